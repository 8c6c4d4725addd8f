// Batch engine: many independent 3D OSEM jobs advanced together, one fused
// launch per step for all of them (continuous batching).  Host-side state
// machine per job: queued -> admitted (buffers, sensitivity) -> passes ->
// final likelihood -> done.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <vector>
#include "internal.h"
#include "../../include/apirl_b200.h"

using apirl::EmJob;
using apirl::SensJob;
using apirl::SubsetSel;
using apirl::UpdJob;

namespace {

apirl_status bfail(apirl_status code, const char* what, cudaError_t e = cudaSuccess) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s%s%s", what, e == cudaSuccess ? "" : ": ", e == cudaSuccess ? "" : cudaGetErrorString(e));
  return apirl_internal_fail(code, buf);
}

#define BK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return bfail(e_ == cudaErrorMemoryAllocation ? APIRL_ERR_OOM : APIRL_ERR_CUDA, #call, e_); \
  } while (0)

size_t count_elem_size(int dtype) { return dtype == APIRL_U16 ? 2 : 4; }

// Passes with at least this many bins get a launch of their own.
#ifndef APIRL_BATCH_OWN_BINS
#define APIRL_BATCH_OWN_BINS (1 << 20)
#endif
constexpr int64_t kOwnLaunchBins = APIRL_BATCH_OWN_BINS;

enum class Stage { Queued, Sens, Passes, Final, Done };

struct Job {
  int64_t id;
  apirl_image_geom img;
  apirl_sino3d_geom sino;
  std::vector<int> mn, mx;
  const void* h_counts = nullptr;  // caller's arrays, read at admission
  const float *h_mult = nullptr, *h_add = nullptr, *h_init = nullptr;
  int dtype;
  int iters, nsub;
  int64_t nbins = 0, nvox = 0, footprint = 0;
  Stage stage = Stage::Queued;
  int pass = 0;
  apirl_projector* p = nullptr;
  void* d_counts = nullptr;
  float *d_mult = nullptr, *d_add = nullptr, *d_x = nullptr, *d_bp = nullptr, *d_sens = nullptr;
  double* d_lik = nullptr;
  std::vector<float> out;
  std::vector<double> lik;
};

int64_t footprint_of(const apirl_image_geom& img, const apirl_sino3d_geom& sino, int dtype, bool mult, bool add,
                     int nsub, int64_t nbins) {
  const int64_t nv = (int64_t)img.nx * img.ny * img.nz;
  int64_t b = nbins * (int64_t)count_elem_size(dtype);
  if (mult) b += nbins * 4;
  if (add) b += nbins * 4;
  const int64_t pv = (int64_t)(img.nx + 2 * apirl::kPad) * (img.ny + 2 * apirl::kPad) * (img.nz + 2 * apirl::kPad);
  b += nv * 4 * (2 + nsub);                               // x, bp, sens per subset
  b += pv * 4 * 4;                                        // padded two-layout image and backprojection copies
  b += (int64_t)sino.n_proj * sino.n_r * 16;              // LOR table
  b += ((nbins + 255) / 256) * 8 + 4096;                  // partials, small tables
  // The geometry-image sparse pass of jobs without factors walks a list of
  // the bins with counts (room for the largest subset).
  if (!mult && !add && sino.n_proj > 0) {
    const int64_t per_angle = nbins / sino.n_proj;
    const int ns = nsub > 0 ? nsub : 1;
    b += per_angle * ((sino.n_proj + ns - 1) / ns) * 4 + 4096;
  }
  return b;
}

}  // namespace

struct apirl_batch {
  int device = 0;
  int64_t budget = 0, used = 0;
  int64_t next_id = 0;
  cudaStream_t st = nullptr;
  std::deque<std::unique_ptr<Job>> queue;
  std::vector<std::unique_ptr<Job>> active;
  std::map<int64_t, std::unique_ptr<Job>> finished;
  // launch scratch
  EmJob* d_em = nullptr; UpdJob* d_upd = nullptr; SensJob* d_sens = nullptr;
  EmJob* h_em = nullptr; UpdJob* h_upd = nullptr; SensJob* h_sens = nullptr;
  int cap_jobs = 0;
  double* d_partials = nullptr;
  int64_t cap_partials = 0;
};

namespace {

void release(Job& j) {
  if (j.p) apirl_projector_destroy(j.p);
  j.p = nullptr;
  cudaFree(j.d_counts); cudaFree(j.d_mult); cudaFree(j.d_add); cudaFree(j.d_x); cudaFree(j.d_bp);
  cudaFree(j.d_sens); cudaFree(j.d_lik);
  j.d_counts = nullptr; j.d_mult = j.d_add = j.d_x = j.d_bp = j.d_sens = nullptr; j.d_lik = nullptr;
}

apirl_status admit(apirl_batch* b, Job& j) {
  j.sino.min_ring_diff = j.mn.data();
  j.sino.max_ring_diff = j.mx.data();
  apirl_status s = apirl_projector_create_3d(&j.img, &j.sino, b->device, &j.p);
  if (s != APIRL_OK) return s;
  const size_t cb = (size_t)j.nbins * count_elem_size(j.dtype);
  BK(cudaMalloc(&j.d_counts, cb));
  BK(cudaMemcpyAsync(j.d_counts, j.h_counts, cb, cudaMemcpyHostToDevice, b->st));
  if (j.h_mult) {
    BK(cudaMalloc(&j.d_mult, j.nbins * sizeof(float)));
    BK(cudaMemcpyAsync(j.d_mult, j.h_mult, j.nbins * sizeof(float), cudaMemcpyHostToDevice, b->st));
  }
  if (j.h_add) {
    BK(cudaMalloc(&j.d_add, j.nbins * sizeof(float)));
    BK(cudaMemcpyAsync(j.d_add, j.h_add, j.nbins * sizeof(float), cudaMemcpyHostToDevice, b->st));
  }
  BK(cudaMalloc(&j.d_x, j.nvox * sizeof(float)));
  BK(cudaMalloc(&j.d_bp, j.nvox * sizeof(float)));
  BK(cudaMalloc(&j.d_sens, j.nvox * j.nsub * sizeof(float)));
  BK(cudaMalloc(&j.d_lik, ((size_t)j.iters * j.nsub + 1) * sizeof(double)));
  if (j.h_init)
    BK(cudaMemcpyAsync(j.d_x, j.h_init, j.nvox * sizeof(float), cudaMemcpyHostToDevice, b->st));
  else
    BK(apirl::launch_fill(j.nvox, j.d_x, 1.f, b->st));
  BK(cudaMemsetAsync(j.d_bp, 0, j.nvox * sizeof(float), b->st));
  BK(cudaMemsetAsync(j.d_sens, 0, j.nvox * j.nsub * sizeof(float), b->st));
  // Without factors each sensitivity image is A_s^T 1, the geometry image of
  // the sparse pass: big jobs' passes then walk only their bins with counts.
  if (!j.h_mult && !j.h_add) {
    s = apirl_projector_set_option(j.p, APIRL_OPT_SPARSE_IMAGE, APIRL_SPARSE_GEOMETRY);
    if (s != APIRL_OK) return s;
  }
  j.stage = Stage::Sens;
  b->used += j.footprint;
  return APIRL_OK;
}

apirl_status ensure_scratch(apirl_batch* b, int njobs, int64_t nblocks) {
  if (njobs > b->cap_jobs) {
    cudaFree(b->d_em); cudaFree(b->d_upd); cudaFree(b->d_sens);
    cudaFreeHost(b->h_em); cudaFreeHost(b->h_upd); cudaFreeHost(b->h_sens);
    int cap = std::max(64, njobs * 2);
    BK(cudaMalloc(&b->d_em, cap * sizeof(EmJob)));
    BK(cudaMalloc(&b->d_upd, cap * sizeof(UpdJob)));
    BK(cudaMalloc(&b->d_sens, cap * sizeof(SensJob)));
    BK(cudaMallocHost(&b->h_em, cap * sizeof(EmJob)));
    BK(cudaMallocHost(&b->h_upd, cap * sizeof(UpdJob)));
    BK(cudaMallocHost(&b->h_sens, cap * sizeof(SensJob)));
    b->cap_jobs = cap;
  }
  if (nblocks > b->cap_partials) {
    cudaFree(b->d_partials);
    int64_t cap = std::max<int64_t>(nblocks, 1 << 16);
    BK(cudaMalloc(&b->d_partials, cap * sizeof(double)));
    b->cap_partials = cap;
  }
  return APIRL_OK;
}

}  // namespace

extern "C" {

int64_t apirl_job_footprint(const apirl_job_desc* job) {
  if (!job) return -1;
  const int n = apirl_sino3d_ring_z(&job->sino, nullptr);
  if (n <= 0) return -1;
  const int64_t nbins = (int64_t)n * job->sino.n_proj * job->sino.n_r;
  return footprint_of(job->img, job->sino, job->counts_dtype, job->h_mult, job->h_add, job->nsubsets, nbins);
}

apirl_status apirl_batch_create(int device, int64_t budget, apirl_batch** out) {
  if (!out || budget <= 0) return bfail(APIRL_ERR_INVALID, "bad arguments");
  int prev = 0;
  cudaGetDevice(&prev);
  BK(cudaSetDevice(device));
  apirl_batch* b = new apirl_batch;
  b->device = device;
  b->budget = budget;
  cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  cudaSetDevice(prev);
  if (e != cudaSuccess) { delete b; return bfail(APIRL_ERR_CUDA, "cudaStreamCreate", e); }
  *out = b;
  return APIRL_OK;
}

void apirl_batch_destroy(apirl_batch* b) {
  if (!b) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->st);
  for (auto& j : b->active) release(*j);
  cudaFree(b->d_em); cudaFree(b->d_upd); cudaFree(b->d_sens); cudaFree(b->d_partials);
  cudaFreeHost(b->h_em); cudaFreeHost(b->h_upd); cudaFreeHost(b->h_sens);
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
  const int nsinos = apirl_sino3d_ring_z(&d->sino, nullptr);
  if (nsinos <= 0) return bfail(APIRL_ERR_INVALID, "segment table yields no sinograms");
  std::unique_ptr<Job> j(new Job);
  j->id = b->next_id++;
  j->img = d->img;
  j->sino = d->sino;
  j->mn.assign(d->sino.min_ring_diff, d->sino.min_ring_diff + d->sino.n_segments);
  j->mx.assign(d->sino.max_ring_diff, d->sino.max_ring_diff + d->sino.n_segments);
  j->nbins = (int64_t)nsinos * d->sino.n_proj * d->sino.n_r;
  j->nvox = (int64_t)d->img.nx * d->img.ny * d->img.nz;
  j->dtype = d->counts_dtype;
  j->h_counts = d->h_counts;
  j->h_mult = d->h_mult;
  j->h_add = d->h_add;
  j->h_init = d->h_init;
  j->iters = d->iters;
  j->nsub = d->nsubsets;
  j->footprint = footprint_of(d->img, d->sino, d->counts_dtype, d->h_mult, d->h_add, d->nsubsets, j->nbins);
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
  // 1. admission: in order, smaller jobs may pass one that does not fit.
  for (auto it = b->queue.begin(); it != b->queue.end();) {
    if (b->used + (*it)->footprint <= b->budget) {
      apirl_status s = admit(b, **it);
      if (s != APIRL_OK) { release(**it); return s; }
      b->active.push_back(std::move(*it));
      it = b->queue.erase(it);
    } else {
      ++it;
    }
  }
  std::vector<Job*> sens, passes, finals, big;
  for (auto& j : b->active) {
    if (j->stage == Stage::Sens) sens.push_back(j.get());
    else if (j->stage == Stage::Passes) {
      // Jobs whose pass fills the GPU on its own run through the single-job
      // fused pass (padded two-layout walk, tuned block size); the rest share
      // one launch.
      if (apirl_projector_num_bins(j->p, j->pass % j->nsub, j->nsub) >= kOwnLaunchBins) big.push_back(j.get());
      else passes.push_back(j.get());
    } else if (j->stage == Stage::Final) finals.push_back(j.get());
  }
  const int njob_max = (int)b->active.size() + 1;
  int64_t em_blocks = 0, upd_blocks = 0, sens_blocks = 0;
  for (Job* j : passes) em_blocks += (apirl_projector_num_bins(j->p, j->pass % j->nsub, j->nsub) + 255) / 256;
  for (Job* j : finals) em_blocks += (j->nbins + 255) / 256;
  apirl_status s = ensure_scratch(b, njob_max, em_blocks);
  if (s != APIRL_OK) return s;
  // 2. sensitivity of newly admitted jobs (all subsets in one pass each).
  int ns = 0;
  for (Job* j : sens) {
    SensJob& S = b->h_sens[ns++];
    S.g = j->p->g; S.t = j->p->t; S.mult = j->d_mult; S.sens = j->d_sens;
    S.blk_begin = sens_blocks; S.nbins = j->nbins; S.nvox = j->nvox; S.nsub = j->nsub;
    sens_blocks += (j->nbins + 255) / 256;
  }
  if (ns) {
    BK(cudaMemcpyAsync(b->d_sens, b->h_sens, ns * sizeof(SensJob), cudaMemcpyHostToDevice, b->st));
    BK(apirl::launch_sens_batch(b->d_sens, ns, sens_blocks, b->st));
    for (Job* j : sens) BK(apirl::launch_force_positive(j->nvox * j->nsub, j->d_sens, b->st));
  }
  // 3. one pass of every running job, and the final likelihood of finishing ones.
  int ne = 0, nu = 0;
  em_blocks = 0;
  for (Job* j : passes) {
    const int sub = j->pass % j->nsub;
    EmJob& E = b->h_em[ne++];
    E.g = j->p->g; E.t = j->p->t;
    E.s.subset = sub; E.s.nsub = j->nsub; E.s.nk = apirl::subset_nproj(j->sino.n_proj, sub, j->nsub);
    E.counts = j->d_counts; E.counts_dtype = j->dtype; E.add = j->d_add; E.x = j->d_x; E.bp = j->d_bp;
    E.lik = j->d_lik + j->pass; E.back = 1; E.lik_mode = 0;
    E.nbins = (int64_t)j->p->t.n_sinos * E.s.nk * j->p->t.n_r;
    E.blk_begin = em_blocks;
    em_blocks += (E.nbins + 255) / 256;
    UpdJob& U = b->h_upd[nu++];
    U.x = j->d_x; U.bp = j->d_bp; U.sens = j->d_sens + (int64_t)sub * j->nvox; U.nvox = j->nvox;
    U.thr = 0.f; U.ge = 1;
    U.blk_begin = upd_blocks;
    upd_blocks += (j->nvox + apirl::kBatchVoxPerBlock - 1) / apirl::kBatchVoxPerBlock;
  }
  for (Job* j : finals) {
    EmJob& E = b->h_em[ne++];
    E.g = j->p->g; E.t = j->p->t;
    E.s.subset = -1; E.s.nsub = 1; E.s.nk = j->sino.n_proj;
    E.counts = j->d_counts; E.counts_dtype = j->dtype; E.add = j->d_add; E.x = j->d_x; E.bp = j->d_bp;
    E.lik = j->d_lik + (int64_t)j->iters * j->nsub; E.back = 0; E.lik_mode = 0;
    E.nbins = j->nbins;
    E.blk_begin = em_blocks;
    em_blocks += (E.nbins + 255) / 256;
  }
  if (ne) {
    BK(cudaMemcpyAsync(b->d_em, b->h_em, ne * sizeof(EmJob), cudaMemcpyHostToDevice, b->st));
    BK(apirl::launch_em_batch(b->d_em, b->h_em, ne, em_blocks, b->d_partials, b->st));
  }
  for (Job* j : big) {
    const int sub = j->pass % j->nsub;
    float* sens_s = j->d_sens + (int64_t)sub * j->nvox;
    apirl_status es = (!j->d_mult && !j->d_add)
                          ? apirl_em_pass_sparse(j->p, j->d_counts, j->dtype, 0, nullptr, j->d_x, j->d_bp, sens_s,
                                                 sens_s, nullptr, nullptr, 0.f, 1, sub, j->nsub, j->d_lik + j->pass,
                                                 b->st)
                          : apirl_em_pass(j->p, j->d_counts, j->dtype, 0, j->d_add, j->d_x, j->d_bp, sens_s, nullptr,
                                          0.f, 1, sub, j->nsub, j->d_lik + j->pass, b->st);
    if (es != APIRL_OK) return es;
  }
  if (nu) {
    BK(cudaMemcpyAsync(b->d_upd, b->h_upd, nu * sizeof(UpdJob), cudaMemcpyHostToDevice, b->st));
    BK(apirl::launch_update_batch(b->d_upd, nu, upd_blocks, b->st));
  }
  BK(cudaStreamSynchronize(b->st));
  // 4. advance and retire.
  for (Job* j : sens) j->stage = j->iters * j->nsub > 0 ? Stage::Passes : Stage::Final;
  for (Job* j : passes) if (++j->pass == j->iters * j->nsub) j->stage = Stage::Final;
  for (Job* j : big) if (++j->pass == j->iters * j->nsub) j->stage = Stage::Final;
  for (Job* j : finals) {
    j->out.resize(j->nvox);
    j->lik.resize((size_t)j->iters * j->nsub + 1);
    BK(cudaMemcpy(j->out.data(), j->d_x, j->nvox * sizeof(float), cudaMemcpyDeviceToHost));
    BK(cudaMemcpy(j->lik.data(), j->d_lik, j->lik.size() * sizeof(double), cudaMemcpyDeviceToHost));
    j->stage = Stage::Done;
  }
  for (auto it = b->active.begin(); it != b->active.end();) {
    if ((*it)->stage == Stage::Done) {
      release(**it);
      b->used -= (*it)->footprint;
      b->finished[(*it)->id] = std::move(*it);
      it = b->active.erase(it);
    } else {
      ++it;
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
