// egpu_server.cpp -- continuous-batching solve server on a host thread (egpu_server_*).
//
// No counterpart in the reference: it extends SolveSystem (SolverUtils.src:7531) to a stream
// of independent systems.  The server owns a context (stream, scratch) and a batch
// (egpu_batch_*).  Callers register mesh patterns once (a resident prototype matrix, as
// Elmer keeps Solver % Matrix across steps) and submit requests: a pattern plus Values and
// RHS from the host, or a pattern plus Poisson material data assembled on the device.
// A worker thread admits queued requests in arrival order while their device footprint fits
// the HBM budget and a batch slot is free, prepares each admitted system (clone of the
// prototype, values or GPU assembly and Dirichlet rows, scaling, ILU0), steps the batch
// (one FP64 refinement check + one chunk of FP32 inner iterations for every resident system),
// and retires converged systems: their solutions are copied to host memory and their slots
// and device memory returned, so requests arriving meanwhile join the next step.
//
// Every GPU call on the server's context happens under one mutex (the worker and pattern
// registration).  Submissions and polls take only the pattern-table and queue locks, so
// they never wait for a GPU step, and callers may use any thread.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/elmergpu.h"
#include "egpu_devmem.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Pattern {
  egpu_mat *proto = nullptr;
  int n = 0;
  long long nnz = 0;
  long long footprint = 0;
  bool mesh = false;
};

enum class St { QUEUED, RESIDENT, DONE };

struct Request {
  long long id = 0;
  int pattern = 0;
  egpu_mat *proto = nullptr;  // the pattern's resident prototype
  int n = 0;                 // rows of the pattern
  double footprint = 0;      // device bytes while resident
  St state = St::QUEUED;
  // inputs: Values + RHS, or Poisson assembly data
  bool assemble = false;
  std::vector<double> values, rhs, elem_k, nodal_k, load;
  std::vector<int> con;
  int symmetric = 0;
  // device state while resident (touched by the worker only)
  egpu_mat *A = nullptr;
  double *rhs_dev = nullptr;
  size_t rhs_cap = 0;
  int rhs_devid = 0;
  int slot = -1;
  // result
  std::vector<double> x;
  egpu_result res{};
  Clock::time_point t_submit, t_admit, t_done;
};

}  // namespace

struct egpu_server {
  int device = 0;
  egpu_params prm{};
  double budget = 0;
  int max_resident = 0;
  egpu_ctx *ctx = nullptr;
  egpu_batch *batch = nullptr;
  std::mutex gpu_mu;  // every call on ctx / batch
  std::mutex pat_mu;  // the pattern table (never held across a GPU call)
  std::vector<Pattern> patterns;
  std::unordered_map<int, int> mesh_nodes, mesh_elems;
  std::mutex mu;      // queue, request table and states, counters (taken before gpu_mu when both)
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<long long, std::unique_ptr<Request>> requests;
  std::unordered_map<int, Request *> by_slot;  // written by the worker under mu
  long long next_id = 1, steps = 0, done = 0;
  double used = 0;
  double t_prepare = 0, t_step = 0, t_retire = 0;  // worker wall time per activity (under mu)
  long long launches = 0;                           // kernel launches of ctx (under mu)
  double bytes_h2d = 0, bytes_d2h = 0;              // request inputs uploaded, solutions read back (under mu)
  long long requeues = 0;                           // admitted requests put back after a failed allocation (under mu)
  bool stop = false;
  std::thread worker;
};

namespace {

// device setup of one admitted request (under gpu_mu); its batch slot or a negative error
int prepare(egpu_server *S, Request *r) {
  int rc = egpu_matrix_clone(r->proto, &r->A);
  if (rc) return rc;
  if (r->assemble) {
    rc = egpu_assemble_poisson(r->A, r->elem_k.empty() ? nullptr : r->elem_k.data(),
                               r->nodal_k.empty() ? nullptr : r->nodal_k.data(),
                               r->load.empty() ? nullptr : r->load.data());
    if (!rc && !r->con.empty())
      rc = egpu_dirichlet(r->A, (int)r->con.size(), r->con.data(), nullptr, r->symmetric);
    if (rc) return rc;
    return egpu_batch_add_matrix(S->batch, r->A, nullptr);
  }
  rc = egpu_matrix_update_values(r->A, r->values.data());
  if (rc) return rc;
  void *q = nullptr;
  if (egpu::dev_alloc(&q, sizeof(double) * r->n, &r->rhs_cap, &r->rhs_devid) != cudaSuccess ||
      !(r->rhs_dev = (double *)q) ||
      cudaMemcpy(r->rhs_dev, r->rhs.data(), sizeof(double) * r->n, cudaMemcpyHostToDevice) != cudaSuccess)
    return EGPU_ERR_ALLOC;
  return egpu_batch_add_matrix(S->batch, r->A, r->rhs_dev);
}

// device memory of a request (under gpu_mu)
void release_device(Request *r) {
  if (r->rhs_dev) egpu::dev_free(r->rhs_dev, r->rhs_cap, r->rhs_devid);
  r->rhs_dev = nullptr;
  if (r->A) egpu_matrix_free(r->A);
  r->A = nullptr;
}

// device and input memory of a request (under gpu_mu)
void release(Request *r) {
  release_device(r);
  std::vector<double>().swap(r->values);
  std::vector<double>().swap(r->rhs);
  std::vector<double>().swap(r->elem_k);
  std::vector<double>().swap(r->nodal_k);
  std::vector<double>().swap(r->load);
  std::vector<int>().swap(r->con);
}

// host bytes a request's preparation copies to the device
double input_bytes(const Request *r) {
  return (double)sizeof(double) * (r->values.size() + r->rhs.size() + r->elem_k.size() + r->nodal_k.size() +
                                   r->load.size()) +
         (double)sizeof(int) * r->con.size();
}

// (under mu)
void finish(egpu_server *S, Request *r, Clock::time_point now) {
  r->t_done = now;
  r->res.seconds = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  r->res.seconds_setup = std::chrono::duration<double>(r->t_admit - r->t_submit).count();
  r->state = St::DONE;
  S->used -= r->footprint;
  S->done++;
}

void work(egpu_server *S) {
  cudaSetDevice(S->device);
  std::vector<int> fin(S->max_resident + 1);
  std::unique_lock<std::mutex> lk(S->mu);
  while (true) {
    S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty() || !S->by_slot.empty(); });
    if (S->stop) break;
    // admission in arrival order: footprint within the budget, within the device memory that
    // is free now (the registered patterns' resident prototypes and other users of the GPU
    // take their share), and a free slot; a request larger than the whole budget still runs,
    // alone
    std::vector<Request *> admit;
    double avail = 0.0;
    {
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) == cudaSuccess)
        avail = (double)fr + (double)egpu_cached_bytes(S->device) - 0.03 * (double)tot;
    }
    double adm_bytes = 0.0;
    while (!S->queue.empty() && (int)(S->by_slot.size() + admit.size()) < S->max_resident) {
      Request *r = S->queue.front();
      const bool alone = S->by_slot.empty() && admit.empty();
      if (!alone && (S->used + r->footprint > S->budget || adm_bytes + r->footprint > avail)) break;
      S->used += r->footprint;
      adm_bytes += r->footprint;
      r->t_admit = Clock::now();
      admit.push_back(r);
      S->queue.pop_front();
    }
    lk.unlock();
    // GPU work: prepare the admitted systems, one step, collect the finished ones
    std::vector<std::pair<Request *, int>> added;
    std::vector<Request *> retired, requeue;
    int step_rc = 0;
    Clock::time_point c0, c1, c2, c3;
    double h2d = 0, d2h = 0;
    long long nl = 0;
    {
      std::lock_guard<std::mutex> g(S->gpu_mu);
      c0 = Clock::now();
      bool placed_any = !S->by_slot.empty();
      for (Request *r : admit) {
        // a device allocation that fails while other requests hold memory puts the request
        // back in the queue, to be admitted again once some of them have retired
        if (!requeue.empty()) {
          requeue.push_back(r);
          continue;
        }
        const int slot = prepare(S, r);
        if (slot < 0 && (slot == EGPU_ERR_ALLOC || slot == EGPU_ERR_CUDA) && placed_any) {
          release_device(r);
          cudaGetLastError();  // an out-of-memory allocation leaves a non-sticky error
          requeue.push_back(r);
          continue;
        }
        h2d += input_bytes(r);
        if (slot < 0) {
          r->res = egpu_result{};
          r->res.info = slot;
          release(r);
        } else {
          placed_any = true;
        }
        added.push_back({r, slot});
      }
      int nf = 0;
      c1 = Clock::now();
      if (egpu_batch_pending(S->batch) > 0) step_rc = egpu_batch_step(S->batch, fin.data(), &nf);
      c2 = Clock::now();
      std::vector<int> done_slots;
      if (step_rc < 0) {  // the batch failed: every resident request ends with the error code
        for (auto &kv : S->by_slot) done_slots.push_back(kv.first);
        for (auto &[r, slot] : added)
          if (slot >= 0) done_slots.push_back(slot);
      } else {
        done_slots.assign(fin.begin(), fin.begin() + nf);
      }
      for (int slot : done_slots) {
        Request *r = nullptr;
        auto it = S->by_slot.find(slot);
        if (it != S->by_slot.end()) r = it->second;
        for (auto &[ra, sa] : added)
          if (sa == slot) r = ra;
        if (!r) continue;
        if (step_rc < 0) {
          r->res = egpu_result{};
          r->res.info = step_rc;
        } else {
          egpu_batch_result(S->batch, slot, &r->res);
          r->x.resize(r->n);
          egpu_batch_solution(S->batch, slot, r->x.data());
          d2h += (double)sizeof(double) * r->n;
        }
        egpu_batch_remove(S->batch, slot);
        release(r);
        retired.push_back(r);
      }
      c3 = Clock::now();
      nl = egpu_kernel_launches(S->ctx);
    }
    lk.lock();
    for (auto it = requeue.rbegin(); it != requeue.rend(); ++it) {
      S->used -= (*it)->footprint;
      S->queue.push_front(*it);
    }
    S->requeues += (long long)requeue.size();
    S->launches = nl;
    S->bytes_h2d += h2d;
    S->bytes_d2h += d2h;
    S->t_prepare += std::chrono::duration<double>(c1 - c0).count();
    S->t_step += std::chrono::duration<double>(c2 - c1).count();
    S->t_retire += std::chrono::duration<double>(c3 - c2).count();
    const auto now = Clock::now();
    for (auto &[r, slot] : added) {
      if (slot < 0) {
        finish(S, r, now);
      } else {
        r->slot = slot;
        r->state = St::RESIDENT;
        S->by_slot[slot] = r;
      }
    }
    for (Request *r : retired) {
      S->by_slot.erase(r->slot);
      finish(S, r, now);
    }
    S->steps++;
    if (!retired.empty() || !added.empty()) S->cv_done.notify_all();
  }
}

// pattern size and footprint (submission never waits for a GPU step)
bool pattern_info(egpu_server *S, int pattern, Pattern &out, int *nnodes = nullptr, int *nelem = nullptr) {
  std::lock_guard<std::mutex> g(S->pat_mu);
  if (pattern < 0 || pattern >= (int)S->patterns.size()) return false;
  out = S->patterns[pattern];
  if (nnodes) *nnodes = S->mesh_nodes.count(pattern) ? S->mesh_nodes[pattern] : 0;
  if (nelem) *nelem = S->mesh_elems.count(pattern) ? S->mesh_elems[pattern] : 0;
  return true;
}

Request *new_request(egpu_server *S, const Pattern &P, int pattern, long long *id) {
  auto r = std::make_unique<Request>();
  r->pattern = pattern;
  r->proto = P.proto;
  r->n = P.n;
  r->footprint = (double)P.footprint;
  r->t_submit = Clock::now();
  Request *p = r.get();
  std::lock_guard<std::mutex> lk(S->mu);
  r->id = S->next_id++;
  *id = r->id;
  S->requests[r->id] = std::move(r);
  return p;
}

void enqueue(egpu_server *S, Request *r) {
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->queue.push_back(r);
  }
  S->cv_work.notify_one();
}

}  // namespace

extern "C" int egpu_server_create(int device, const egpu_params *prm, double hbm_budget_bytes, int chunk_iters,
                                  int max_resident, egpu_server **out) {
  if (!prm || !out || hbm_budget_bytes <= 0 || max_resident < 1) return EGPU_ERR_ARG;
  auto *S = new egpu_server;
  S->device = device;
  S->prm = *prm;
  S->budget = hbm_budget_bytes;
  S->max_resident = std::min(max_resident, 512);
  int rc = egpu_create(device, &S->ctx);
  if (!rc) rc = egpu_batch_create(S->ctx, prm, &S->batch);
  if (!rc && chunk_iters > 0) rc = egpu_batch_set_chunk(S->batch, chunk_iters);
  if (!rc) rc = egpu_batch_set_latency_mode(S->batch, 1);  // retire each request as it finishes
  if (rc) {
    if (S->batch) egpu_batch_free(S->batch);
    if (S->ctx) egpu_destroy(S->ctx);
    delete S;
    return rc;
  }
  S->worker = std::thread(work, S);
  *out = S;
  return EGPU_OK;
}

extern "C" int egpu_server_pattern(egpu_server *S, int n, const int *rows, const int *cols, const int *diag,
                                   int *pattern) {
  if (!S || !rows || !cols || !diag || !pattern || n < 1) return EGPU_ERR_ARG;
  const long long nnz = (long long)rows[n] - rows[0];
  if (nnz < 1) return EGPU_ERR_ARG;
  std::vector<double> zero(nnz, 0.0);
  Pattern P;
  P.n = n;
  P.nnz = nnz;
  {
    std::lock_guard<std::mutex> g(S->gpu_mu);
    int rc = egpu_matrix_bind(S->ctx, n, rows, cols, diag, zero.data(), &P.proto);
    if (!rc) rc = egpu_matrix_prepare(P.proto, &S->prm);
    if (rc) {
      if (P.proto) egpu_matrix_free(P.proto);
      return rc;
    }
    P.footprint = egpu_matrix_footprint(P.proto, S->prm.precond);
  }
  std::lock_guard<std::mutex> g(S->pat_mu);
  S->patterns.push_back(P);
  *pattern = (int)S->patterns.size() - 1;
  return EGPU_OK;
}

extern "C" int egpu_server_pattern_mesh(egpu_server *S, int pattern, int nnodes, const double *xyz, int cdim,
                                        int nelem, int code, const int *elem_nodes, const int *perm, int dofs) {
  Pattern P;
  if (!S || !pattern_info(S, pattern, P)) return EGPU_ERR_ARG;
  int rc;
  {
    std::lock_guard<std::mutex> g(S->gpu_mu);
    rc = egpu_assembly_bind(P.proto, nnodes, xyz, cdim, nelem, code, elem_nodes, perm, dofs);
  }
  if (!rc) {
    std::lock_guard<std::mutex> g(S->pat_mu);
    S->patterns[pattern].mesh = true;
    S->mesh_nodes[pattern] = nnodes;
    S->mesh_elems[pattern] = nelem;
  }
  return rc;
}

extern "C" int egpu_server_submit(egpu_server *S, int pattern, const double *values, const double *rhs,
                                  long long *request) {
  Pattern P;
  if (!S || !values || !rhs || !request || !pattern_info(S, pattern, P)) return EGPU_ERR_ARG;
  Request *r = new_request(S, P, pattern, request);
  r->values.assign(values, values + P.nnz);
  r->rhs.assign(rhs, rhs + P.n);
  enqueue(S, r);
  return EGPU_OK;
}

extern "C" int egpu_server_submit_poisson(egpu_server *S, int pattern, const double *elem_k, const double *nodal_k,
                                          const double *load, int ncon, const int *con_rows, int symmetric,
                                          long long *request) {
  Pattern P;
  int nnodes = 0, nelem = 0;
  if (!S || !request || ncon < 0 || (ncon > 0 && !con_rows) || !pattern_info(S, pattern, P, &nnodes, &nelem))
    return EGPU_ERR_ARG;
  if (!P.mesh) return EGPU_ERR_STATE;
  Request *r = new_request(S, P, pattern, request);
  r->assemble = true;
  if (elem_k) r->elem_k.assign(elem_k, elem_k + nelem);
  if (nodal_k) r->nodal_k.assign(nodal_k, nodal_k + nnodes);
  if (load) r->load.assign(load, load + nnodes);
  if (ncon) r->con.assign(con_rows, con_rows + ncon);
  r->symmetric = symmetric;
  enqueue(S, r);
  return EGPU_OK;
}

// 1: done (x, res filled; the request is released), 0: pending, < 0: unknown request
extern "C" int egpu_server_poll(egpu_server *S, long long request, double *x, egpu_result *res) {
  if (!S) return EGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->requests.find(request);
  if (it == S->requests.end()) return EGPU_ERR_ARG;
  Request *r = it->second.get();
  if (r->state != St::DONE) return 0;
  if (x && !r->x.empty()) std::memcpy(x, r->x.data(), r->x.size() * sizeof(double));
  if (res) *res = r->res;
  S->requests.erase(it);
  return 1;
}

// as egpu_server_poll, blocking up to timeout_s seconds (EGPU_ERR_TIMEOUT when it expires)
extern "C" int egpu_server_wait(egpu_server *S, long long request, double timeout_s, double *x,
                                egpu_result *res) {
  if (!S) return EGPU_ERR_ARG;
  {
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->requests.find(request);
    if (it == S->requests.end()) return EGPU_ERR_ARG;
    Request *r = it->second.get();
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    if (!S->cv_done.wait_until(lk, until, [&] { return r->state == St::DONE; })) return EGPU_ERR_TIMEOUT;
  }
  return egpu_server_poll(S, request, x, res);
}

extern "C" int egpu_server_info(egpu_server *S, egpu_server_stats *st) {
  if (!S || !st) return EGPU_ERR_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  st->queued = (long long)S->queue.size();
  st->resident = (long long)S->by_slot.size();
  st->done = S->done;
  st->steps = S->steps;
  st->used_bytes = S->used;
  st->seconds_prepare = S->t_prepare;
  st->seconds_step = S->t_step;
  st->seconds_retire = S->t_retire;
  st->kernel_launches = S->launches;
  st->bytes_h2d = S->bytes_h2d;
  st->bytes_d2h = S->bytes_d2h;
  st->requeues = S->requeues;
  return EGPU_OK;
}

extern "C" void egpu_server_free(egpu_server *S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  std::lock_guard<std::mutex> g(S->gpu_mu);
  for (auto &kv : S->by_slot) {
    egpu_batch_remove(S->batch, kv.first);
    release(kv.second);
  }
  S->requests.clear();
  egpu_batch_free(S->batch);
  for (Pattern &P : S->patterns) egpu_matrix_free(P.proto);  // no other thread runs now
  egpu_destroy(S->ctx);
  delete S;
}
