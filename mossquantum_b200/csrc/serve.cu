// Serving loop: continuous batching of ansatz evaluations and adjoint gradients.
//
// The reference evaluates one objective per call (evaluate / value_and_gradient,
// src/api/objectives.jl:15-244, src/differentiation/objectives.jl:183-296) and batches only
// samples that share n and theta (src/states/batch_state_vector.jl). Here a scheduler thread
// keeps a population of independent requests resident in HBM and advances all of them on
// every iteration:
//   * admission: queued requests enter in arrival order while the server's byte budget holds
//     their state (16*2^n pure, 16*4^n density) plus gradient buffers and checkpoints;
//   * forward: requests with the same block circuit and kind live in one contiguous pool of
//     samples; one iteration applies one block repetition to the whole pool with the fused
//     pass kernels and per-sample parameters (each request at its own layer);
//   * a request whose layers are done gets <H> from the expectation kernel on its slot and
//     leaves the pool (the last sample moves into its slot, keeping the pool contiguous);
//     gradient requests seed delta = 2H psi (pure) or H (density) and then run one reverse
//     layer per iteration (specialised dual-state passes for pure states, two-level
//     recomputation of channel inputs for density matrices);
//   * everything of an iteration is queued on the library stream; the thread then waits on
//     one event without holding the library lock, and harvests results from pinned memory.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "internal.h"
#include "jit.h"

using namespace mb;

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

enum Phase { PH_PENDING = 0, PH_FORWARD = 1, PH_REVERSE = 2, PH_DONE = 3 };

struct Class;

struct Req {
  uint64_t ticket = 0;
  Class* cls = nullptr;
  mb_observable obs = nullptr;
  int gradient = 0, L = 0;
  std::vector<double> theta;    // L rows of nslots values
  double t_submit = 0, t_admit = 0, t_done = 0;
  int phase = PH_PENDING;
  int slot = -1;                // pool slot during the forward phase
  int layer = 0;                // forward: next layer; reverse: next layer to undo
  int iters = 0;
  size_t extra = 0;             // bytes charged beyond the pool slot
  double2* y = nullptr;         // pure gradient: state being uncomputed
  double2* delta = nullptr;     // gradient: adjoint state
  double* d_grad = nullptr;     // L * nslots
  std::vector<double2*> ckpt;   // density gradient: state before each layer
  std::vector<double2*> scratch;
  int status = MB_OK;
  std::string err;
  double value[2] = {0, 0};
  std::vector<double> grad;
  int res_idx = -1;             // this iteration's slot in the result buffer
  size_t grad_off = SIZE_MAX;   // this iteration's offset of the gradient in the pinned arena
  bool finishing = false;
};

struct Class {
  uint64_t uid = 0;             // block circuit uid
  bool dm = false;
  int n = 0;
  int64_t elems = 0;
  size_t sbytes = 0;
  mb_circuit priv = nullptr;    // private clone: own matrix table, parameters, schedules
  double2* pool = nullptr;
  int cap = 0;
  std::vector<Req*> slots;      // forward-phase requests, slot i holds sample i
  int fused_adjoint = 1;        // 1 try the specialised reverse passes, 0 plain
  int dm_scratch = 0;           // density reverse: scratch states per request
  double* d_theta = nullptr;
  size_t theta_cap = 0;
};

}  // namespace

struct mb_server_s {
  size_t budget = 0, used = 0, peak = 0;
  int max_active = 4096;
  std::thread th;
  std::mutex qmu;
  std::condition_variable qcv, done_cv;
  std::deque<Req*> incoming;                       // qmu
  std::unordered_map<uint64_t, Req*> finished;     // qmu
  std::unordered_set<uint64_t> inflight;           // qmu
  uint64_t next_ticket = 1;                        // qmu
  bool stop = false;                               // qmu
  std::vector<double> lat;                         // qmu
  uint64_t submitted = 0, completed = 0, failed = 0, iterations = 0;
  double t_first = -1, t_last = 0;
  double jit_ms0 = 0;         // compile counters at start / last stats reset
  uint64_t jit_n0 = 0;
  int n_active = 0, n_pending = 0;                 // qmu (mirrors of loop-owned counts)
  // loop-owned
  std::deque<Req*> pending;
  std::vector<Req*> active;
  std::vector<std::unique_ptr<Class>> classes;     // g_mu
  double* arena = nullptr;                         // pinned per-iteration staging
  size_t arena_cap = 0;                            // doubles
  double2* d_res = nullptr;
  int res_cap = 0;
  cudaEvent_t ev = nullptr;
  bool fatal = false;
};

namespace {

int g_servers_running = 0;  // g_mu

Class* find_class(mb_server S, mb_circuit block, bool dm) {
  for (auto& c : S->classes)
    if (c->uid == block->uid && c->dm == dm) return c.get();
  return nullptr;
}

int make_class(mb_server S, mb_circuit block, bool dm, Class** out) {
  std::unique_ptr<Class> c(new Class());
  c->uid = block->uid;
  c->dm = dm;
  c->n = block->n;
  c->elems = dm ? (int64_t(1) << (2 * block->n)) : (int64_t(1) << block->n);
  c->sbytes = sizeof(double2) * size_t(c->elems);  // samples back to back, as the batch kernels index them
  int rc = circuit_clone(block, &c->priv);
  if (rc) return rc;
  if (dm) {
    int m = 1;
    dm_reverse_plan(c->priv, &m, &c->dm_scratch);
  }
  *out = c.get();
  S->classes.push_back(std::move(c));
  return MB_OK;
}

size_t extra_bytes(const Req* r) {
  const Class* c = r->cls;
  if (!r->gradient) return 0;
  const size_t g = round256(sizeof(double) * std::max<size_t>(1, size_t(r->L) * c->priv->nslots));
  if (!c->dm) return 2 * c->sbytes + g;
  return c->sbytes * (1 + size_t(r->L) + size_t(c->dm_scratch)) + g;
}

void charge(mb_server S, size_t b) {
  S->used += b;
  S->peak = std::max(S->peak, S->used);
}

void release_request_memory(mb_server S, Req* r) {
  dev_free(r->y);
  dev_free(r->delta);
  dev_free(r->d_grad);
  for (double2* p : r->ckpt) dev_free(p);
  for (double2* p : r->scratch) dev_free(p);
  r->y = r->delta = nullptr;
  r->d_grad = nullptr;
  r->ckpt.clear();
  r->scratch.clear();
  S->used -= r->extra;
  r->extra = 0;
}

int alloc_request_memory(Req* r) {
  const Class* c = r->cls;
  if (!r->gradient) return MB_OK;
  int rc;
  const size_t g = sizeof(double) * std::max<size_t>(1, size_t(r->L) * c->priv->nslots);
  if ((rc = dev_alloc((void**)&r->delta, c->sbytes)) || (rc = dev_alloc((void**)&r->d_grad, g))) return rc;
  if (!c->dm) return dev_alloc((void**)&r->y, c->sbytes);
  r->ckpt.assign(r->L, nullptr);
  for (int l = 0; l < r->L; ++l)
    if ((rc = dev_alloc((void**)&r->ckpt[l], c->sbytes))) return rc;
  r->scratch.assign(c->dm_scratch, nullptr);
  for (int i = 0; i < c->dm_scratch; ++i)
    if ((rc = dev_alloc((void**)&r->scratch[i], c->sbytes))) return rc;
  return MB_OK;
}

// Resizes a class pool to `cap` samples, keeping the active prefix.
int resize_pool(mb_server S, Class* c, int cap) {
  double2* np = nullptr;
  if (cap > 0) {
    int rc = dev_alloc((void**)&np, c->sbytes * size_t(cap));
    if (rc) return rc;
    const size_t keep = c->sbytes * std::min<size_t>(c->slots.size(), size_t(cap));
    if (keep) MB_CHECK_CUDA(cudaMemcpyAsync(np, c->pool, keep, cudaMemcpyDeviceToDevice, g_ctx.stream));
  }
  dev_free(c->pool);
  S->used -= c->sbytes * size_t(c->cap);
  c->pool = np;
  c->cap = cap;
  charge(S, c->sbytes * size_t(cap));
  return MB_OK;
}

void fail(Req* r, int code, const std::string& msg) {
  r->status = code;
  r->err = msg;
  r->finishing = true;
}

std::string last_error_copy() { return std::string(mb_last_error()); }

// Removes a forward-phase request from its pool: the last sample moves into its slot.
int leave_pool(Class* c, Req* r) {
  const int s = r->slot, last = int(c->slots.size()) - 1;
  if (s < 0) return MB_OK;
  if (s != last) {
    Req* m = c->slots[last];
    MB_CHECK_CUDA(cudaMemcpyAsync(c->pool + int64_t(s) * (c->sbytes / sizeof(double2)),
                                  c->pool + int64_t(last) * (c->sbytes / sizeof(double2)), c->sbytes,
                                  cudaMemcpyDeviceToDevice, g_ctx.stream));
    c->slots[s] = m;
    m->slot = s;
  }
  c->slots.pop_back();
  r->slot = -1;
  return MB_OK;
}

double2* slot_ptr(Class* c, int s) { return c->pool + int64_t(s) * int64_t(c->sbytes / sizeof(double2)); }

// ---- admission ---------------------------------------------------------------------------
void admit(mb_server S) {
  while (!S->pending.empty()) {
    Req* r = S->pending.front();
    Class* c = r->cls;
    if (int(S->active.size()) >= S->max_active) return;
    const size_t extra = extra_bytes(r);
    const int need_cap = int(c->slots.size()) + 1;
    const size_t grow_min = need_cap > c->cap ? c->sbytes * size_t(need_cap - c->cap) : 0;
    if (S->used + extra + grow_min > S->budget) {
      if (S->active.empty()) {
        // Nothing will free memory: the request cannot fit even alone.
        if (extra + c->sbytes > S->budget) {
          S->pending.pop_front();
          char buf[160];
          snprintf(buf, sizeof(buf), "request needs %zu bytes, the server budget is %zu", extra + c->sbytes, S->budget);
          fail(r, MB_ENOMEM_BUDGET, buf);
          S->active.push_back(r);  // harvested as failed this iteration
          continue;
        }
        // Only idle pools hold the memory: release them and retry.
        bool freed = false;
        for (auto& cl : S->classes)
          if (cl->slots.empty() && cl->cap > 0 && resize_pool(S, cl.get(), 0) == MB_OK) freed = true;
        if (freed) continue;
      }
      return;
    }
    int rc = MB_OK;
    if (need_cap > c->cap) {
      const size_t room = S->budget - S->used - extra;
      const int want = std::max(need_cap, std::max(4, 2 * c->cap));
      const int by_room = c->cap + int(std::min<size_t>(room / c->sbytes, size_t(1) << 20));
      rc = resize_pool(S, c, std::max(need_cap, std::min(want, by_room)));
    }
    if (!rc) {
      rc = alloc_request_memory(r);
      if (!rc) {
        r->extra = extra;
        charge(S, extra);
      } else {
        r->extra = 0;
        release_request_memory(S, r);
      }
    }
    if (rc) {
      if (S->active.empty()) {
        S->pending.pop_front();
        fail(r, rc, last_error_copy());
        S->active.push_back(r);
        continue;
      }
      return;  // wait for memory to free up
    }
    S->pending.pop_front();
    r->slot = int(c->slots.size());
    c->slots.push_back(r);
    r->phase = PH_FORWARD;
    r->layer = 0;
    r->t_admit = now_ms();
    if ((rc = launch_set_basis(slot_ptr(c, r->slot), c->elems, 1, 0, g_ctx.stream))) {
      fail(r, rc, last_error_copy());
      leave_pool(c, r);
    }
    S->active.push_back(r);
  }
}

int ensure_theta(Class* c, size_t count) {
  if (count <= c->theta_cap) return MB_OK;
  const size_t cap = std::max<size_t>(count, 2 * c->theta_cap);
  dev_free(c->d_theta);
  c->d_theta = nullptr;
  c->theta_cap = 0;
  int rc = dev_alloc((void**)&c->d_theta, sizeof(double) * cap);
  if (!rc) c->theta_cap = cap;
  return rc;
}

int ensure_table_rows(Class* c, int rows) {
  mb_circuit p = c->priv;
  if (rows <= p->table_rows) return MB_OK;
  const int nr = std::max(rows, 2 * p->table_rows);
  double2* t = nullptr;
  int rc = dev_alloc((void**)&t, sizeof(double2) * p->table_elems * nr);
  if (rc) return rc;
  MB_CHECK_CUDA(cudaMemcpyAsync(t, p->fixed_table.data(), sizeof(double2) * p->table_elems, cudaMemcpyHostToDevice,
                                g_ctx.stream));
  dev_free(p->d_table);
  p->d_table = t;
  p->table_rows = nr;
  return MB_OK;
}

// Binds `rows` parameter rows (already in the pinned arena at h) into the class's table.
int bind_rows(Class* c, const double* h, int rows) {
  mb_circuit p = c->priv;
  int rc;
  if ((rc = ensure_table_rows(c, rows))) return rc;
  if (p->binds.empty()) return MB_OK;
  const size_t cnt = size_t(rows) * p->nslots;
  if (cnt) {
    if ((rc = ensure_theta(c, cnt))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(c->d_theta, h, sizeof(double) * cnt, cudaMemcpyHostToDevice, g_ctx.stream));
  }
  return launch_bind(p->d_binds, int(p->binds.size()), c->d_theta, p->nslots, rows, p->d_table, p->table_elems,
                     g_ctx.stream);
}

// ---- one iteration -------------------------------------------------------------------------
// Queues the iteration's work; returns the offset of the result block in the arena.
void issue(mb_server S, size_t* res_off, int* nres) {
  cudaStream_t st = g_ctx.stream;
  // Arena: parameter rows, result pairs and gradients of this iteration.
  size_t need = 16;
  for (Req* r : S->active) {
    const size_t ns = r->cls->priv->nslots;
    need += ns + 2 + (r->gradient ? size_t(r->L) * ns : 0);
  }
  if (need > S->arena_cap) {
    if (S->arena) cudaFreeHost(S->arena);
    S->arena = nullptr;
    S->arena_cap = 0;
    if (cudaMallocHost((void**)&S->arena, sizeof(double) * need * 2) != cudaSuccess) {
      cudaGetLastError();
      for (Req* r : S->active) fail(r, MB_EDEVICE, "pinned staging allocation failed");
      S->fatal = true;
      return;
    }
    S->arena_cap = need * 2;
  }
  if (int(S->active.size()) > S->res_cap) {
    dev_free(S->d_res);
    S->d_res = nullptr;
    S->res_cap = 0;
    const int cap = std::max<int>(int(S->active.size()) * 2, 64);
    if (dev_alloc((void**)&S->d_res, sizeof(double2) * cap) != MB_OK) {
      for (Req* r : S->active) fail(r, MB_ENOMEM_BUDGET, "result buffer allocation failed");
      return;
    }
    S->res_cap = cap;
  }
  size_t off = 0;
  int nr = 0;
  // Forward: one block repetition for every pool.
  for (auto& cu : S->classes) {
    Class* c = cu.get();
    const int a = int(c->slots.size());
    if (a == 0) continue;
    mb_circuit p = c->priv;
    int rc = MB_OK;
    for (Req* r : c->slots)
      if (r->gradient && c->dm && !rc)
        if (cudaMemcpyAsync(r->ckpt[r->layer], slot_ptr(c, r->slot), c->sbytes, cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess)
          rc = MB_EDEVICE;
    double* h = S->arena + off;
    for (int s = 0; s < a; ++s) {
      const Req* r = c->slots[s];
      if (p->nslots) std::memcpy(h + size_t(s) * p->nslots, r->theta.data() + size_t(r->layer) * p->nslots,
                                 sizeof(double) * p->nslots);
    }
    off += size_t(a) * p->nslots;
    if (!rc) rc = bind_rows(c, h, a);
    if (!rc) {
      mb_state_s view;
      view.kind = c->dm ? MB_BATCH_DENSITY : MB_BATCH_PURE;
      view.n = c->n;
      view.batch = a;
      view.dim = int64_t(1) << c->n;
      view.elems = c->elems;
      view.d = c->pool;
      view.bytes = c->sbytes * a;
      rc = p->ops.empty() ? MB_OK : apply_fused(p, &view, p->table_elems);
    }
    if (rc) {
      const std::string msg = last_error_copy();
      std::vector<Req*> all = c->slots;
      for (Req* r : all) {
        fail(r, rc, msg);
        leave_pool(c, r);
      }
      if (rc == MB_EDEVICE) S->fatal = true;
      continue;
    }
    for (Req* r : c->slots) {
      ++r->layer;
      ++r->iters;
    }
  }
  // Requests whose layers are done: <H>, then leave the pool (gradients: seed the reverse).
  for (auto& cu : S->classes) {
    Class* c = cu.get();
    std::vector<Req*> done;
    for (Req* r : c->slots)
      if (r->layer >= r->L) done.push_back(r);
    for (Req* r : done) {
      mb_state_s v1;
      v1.kind = c->dm ? MB_DENSITY : MB_PURE;
      v1.n = c->n;
      v1.batch = 1;
      v1.dim = int64_t(1) << c->n;
      v1.elems = c->elems;
      v1.d = slot_ptr(c, r->slot);
      v1.bytes = c->sbytes;
      r->res_idx = nr++;
      double2* out = S->d_res + r->res_idx;
      int rc = (!c->dm && r->obs->pauli_ok) ? expect_pauli(r->obs, &v1, out) : expect_keys(r->obs, &v1, out);
      if (!rc && r->gradient) {
        const int64_t L_ns = int64_t(r->L) * c->priv->nslots;
        if (L_ns) rc = cudaMemsetAsync(r->d_grad, 0, sizeof(double) * L_ns, st) == cudaSuccess ? MB_OK : MB_EDEVICE;
        if (!rc && !c->dm) {
          // delta = 2 H psi for Hermitian H (expectation.jl:4-73)
          rc = cudaMemcpyAsync(r->y, v1.d, c->sbytes, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? MB_OK : MB_EDEVICE;
          bool seeded = false;
          if (!rc && r->obs->pauli_ok) rc = pauli_apply(r->obs, r->y, r->delta, c->n, 1, 2.0, &seeded);
          if (!rc && !seeded) {
            rc = observable_apply(r->obs, r->y, r->delta, c->n, 0, 1);
            if (!rc) rc = launch_scale(r->delta, c->elems, 2.0, st);
          }
        } else if (!rc) {
          // delta = H as a density matrix (H applied to the identity)
          rc = launch_identity_density(r->scratch[0], c->n, 1, st);
          if (!rc) rc = observable_apply(r->obs, r->scratch[0], r->delta, c->n, 1, 1);
        }
        if (!rc) {
          r->phase = PH_REVERSE;
          r->layer = r->L - 1;
        }
      } else if (!rc) {
        r->finishing = true;
      }
      if (rc) {
        fail(r, rc, last_error_copy());
        if (rc == MB_EDEVICE) S->fatal = true;
      }
      leave_pool(c, r);
    }
  }
  // Reverse: one layer for every gradient request in its reverse phase.
  for (Req* r : S->active) {
    if (r->phase != PH_REVERSE || r->finishing) continue;
    Class* c = r->cls;
    mb_circuit p = c->priv;
    double* h = S->arena + off;
    if (p->nslots) std::memcpy(h, r->theta.data() + size_t(r->layer) * p->nslots, sizeof(double) * p->nslots);
    off += p->nslots;
    int rc = bind_rows(c, h, 1);
    double* g = r->d_grad + size_t(r->layer) * p->nslots;
    if (!rc && !c->dm) {
      bool used = false;
      rc = reverse_pure_single(p, c->n, r->y, r->delta, g, c->fused_adjoint == 1, &used);
      if (!rc && !used) c->fused_adjoint = 0;
    } else if (!rc) {
      rc = reverse_dm_single(p, c->n, r->ckpt[r->layer], r->delta, g, r->scratch.data());
    }
    ++r->iters;
    if (rc) {
      fail(r, rc, last_error_copy());
      if (rc == MB_EDEVICE) S->fatal = true;
      continue;
    }
    if (--r->layer < 0) {
      const size_t cnt = size_t(r->L) * p->nslots;
      r->grad_off = off;
      if (cnt && cudaMemcpyAsync(S->arena + off, r->d_grad, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st) !=
                     cudaSuccess) {
        fail(r, MB_EDEVICE, "gradient download failed");
        S->fatal = true;
        continue;
      }
      off += cnt;
      r->finishing = true;
    }
  }
  *res_off = off;
  *nres = nr;
  if (nr && cudaMemcpyAsync(S->arena + off, S->d_res, sizeof(double2) * nr, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    S->fatal = true;
}

void server_loop(mb_server S) {
  cudaSetDevice(g_ctx.device);
  // Expectation passes built on this thread stay on the interpreter kernel: a request never
  // waits for NVRTC on an observable first met here.
  pauli_allow_compile(false);
  for (;;) {
    bool stopping;
    {
      std::unique_lock<std::mutex> lk(S->qmu);
      S->qcv.wait(lk, [&] { return S->stop || !S->incoming.empty() || !S->pending.empty() || !S->active.empty(); });
      while (!S->incoming.empty()) {
        S->pending.push_back(S->incoming.front());
        S->incoming.pop_front();
      }
      stopping = S->stop;
      if (stopping || S->fatal) {
        for (Req* r : S->pending) {
          r->status = S->fatal ? MB_EDEVICE : MB_EINVAL;
          r->err = S->fatal ? "the server stopped after a device error" : "the server was stopped";
          r->t_done = now_ms();
          S->finished[r->ticket] = r;
          S->inflight.erase(r->ticket);
          ++S->failed;
        }
        S->pending.clear();
        S->n_pending = 0;
        if (S->active.empty()) {
          S->done_cv.notify_all();
          break;
        }
        S->done_cv.notify_all();
      }
    }
    size_t res_off = 0;
    int nres = 0;
    {
      std::lock_guard<std::recursive_mutex> g(g_mu);
      // Pools left with no requests give their memory back.
      for (auto& c : S->classes)
        if (c->slots.empty() && c->cap > 0) resize_pool(S, c.get(), 0);
        else if (c->cap > 8 && int(c->slots.size()) * 4 < c->cap) resize_pool(S, c.get(), std::max(4, 2 * int(c->slots.size())));
      if (!stopping && !S->fatal) admit(S);
      issue(S, &res_off, &nres);
      if (cudaEventRecord(S->ev, g_ctx.stream) != cudaSuccess) S->fatal = true;
    }
    cudaError_t e = cudaEventSynchronize(S->ev);
    if (e != cudaSuccess) {
      S->fatal = true;
      for (Req* r : S->active) fail(r, MB_EDEVICE, cudaGetErrorString(e));
    }
    // Harvest.
    std::vector<Req*> keep, out;
    for (Req* r : S->active) {
      if (r->res_idx >= 0 && e == cudaSuccess) {
        r->value[0] = S->arena[res_off + 2 * size_t(r->res_idx)];
        r->value[1] = S->arena[res_off + 2 * size_t(r->res_idx) + 1];
      }
      r->res_idx = -1;
      if (r->finishing && r->status == MB_OK && r->grad_off != SIZE_MAX) {
        const size_t cnt = size_t(r->L) * r->cls->priv->nslots;
        r->grad.assign(S->arena + r->grad_off, S->arena + r->grad_off + cnt);
      }
      r->grad_off = SIZE_MAX;
      (r->finishing ? out : keep).push_back(r);
    }
    S->active.swap(keep);
    if (!out.empty()) {
      std::lock_guard<std::recursive_mutex> g(g_mu);
      for (Req* r : out) {
        if (r->slot >= 0) leave_pool(r->cls, r);
        release_request_memory(S, r);
      }
    }
    {
      std::lock_guard<std::mutex> lk(S->qmu);
      const double t = now_ms();
      for (Req* r : out) {
        r->phase = PH_DONE;
        r->t_done = t;
        if (r->status == MB_OK) {
          ++S->completed;
          S->lat.push_back(r->t_done - r->t_submit);
          S->t_last = t;
        } else {
          ++S->failed;
        }
        S->finished[r->ticket] = r;
        S->inflight.erase(r->ticket);
      }
      ++S->iterations;
      S->n_active = int(S->active.size());
      S->n_pending = int(S->pending.size());
    }
    if (!out.empty()) S->done_cv.notify_all();
  }
}

int copy_result(Req* r, mb_result* res, double* grad, size_t ngrad) {
  if (res) {
    std::memset(res, 0, sizeof(*res));
    res->status = r->status;
    res->iterations = r->iters;
    res->value[0] = r->value[0];
    res->value[1] = r->value[1];
    res->latency_ms = r->t_done - r->t_submit;
    res->queue_ms = (r->t_admit > 0 ? r->t_admit : r->t_done) - r->t_submit;
    snprintf(res->error, sizeof(res->error), "%s", r->err.c_str());
  }
  if (grad && r->status == MB_OK && !r->grad.empty()) {
    if (ngrad < r->grad.size()) {
      set_error("gradient buffer holds %zu values, the request has %zu", ngrad, r->grad.size());
      return MB_EINVAL;
    }
    std::memcpy(grad, r->grad.data(), sizeof(double) * r->grad.size());
  }
  return MB_OK;
}

}  // namespace

extern "C" int mb_server_start(const mb_server_config* cfg, mb_server* out) {
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (int rc = check_init()) return rc;
  if (!out) return MB_EINVAL;
  std::unique_ptr<mb_server_s> S(new mb_server_s());
  jit_stats(&S->jit_ms0, &S->jit_n0, nullptr);
  const size_t left = g_ctx.budget > g_ctx.used ? g_ctx.budget - g_ctx.used : 0;
  S->budget = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : size_t(double(left) * 0.95);
  if (S->budget > left) {
    set_error("server budget %zu exceeds the %zu bytes the library budget leaves", S->budget, left);
    return MB_ENOMEM_BUDGET;
  }
  if (cfg && cfg->max_active < 0) return MB_EINVAL;
  if (cfg && cfg->max_active > 0) S->max_active = cfg->max_active;
  MB_CHECK_CUDA(cudaEventCreateWithFlags(&S->ev, cudaEventDisableTiming));
  mb_server s = S.release();
  try {
    s->th = std::thread(server_loop, s);
  } catch (...) {
    cudaEventDestroy(s->ev);
    delete s;
    set_error("could not start the scheduler thread");
    return MB_EDEVICE;
  }
  ++g_servers_running;
  *out = s;
  return MB_OK;
}

extern "C" int mb_submit(mb_server S, const mb_request* q, uint64_t* ticket) {
  if (!S || !q || !ticket) return MB_EINVAL;
  std::unique_ptr<Req> r(new Req());
  {
    std::lock_guard<std::recursive_mutex> g(g_mu);
    if (int rc = check_init()) return rc;
    mb_circuit b = q->block;
    if (!b || !q->observable) {
      set_error("a request needs a block circuit and an observable");
      return MB_EINVAL;
    }
    if (q->kind != MB_PURE && q->kind != MB_DENSITY) {
      set_error("request kind must be MB_PURE or MB_DENSITY");
      return MB_EINVAL;
    }
    const bool dm = q->kind == MB_DENSITY;
    if (q->repeats < 1 || q->repeats > (1 << 20)) {
      set_error("repeats must be in 1..2^20");
      return MB_EINVAL;
    }
    if (b->n > (dm ? 15 : 32) || (dm && 2 * b->n > 30)) {
      set_error("%d qubits out of range for a %s request", b->n, dm ? "density-matrix" : "pure");
      return MB_EINVAL;
    }
    if (b->has_channel && !dm) {
      set_error("a block with channels needs a density-matrix request");
      return MB_EUNSUPPORTED;
    }
    const size_t nt = size_t(q->repeats) * b->nslots;
    if (q->ntheta != nt || (nt && !q->theta)) {
      set_error("expected %zu parameter values (%d layers x %d), got %zu", nt, q->repeats, b->nslots, q->ntheta);
      return MB_EINVAL;
    }
    for (size_t i = 0; i < nt; ++i)
      if (!std::isfinite(q->theta[i])) {
        set_error("parameter values must be finite");
        return MB_EINVAL;
      }
    mb_state_s probe;
    probe.kind = q->kind;
    probe.n = b->n;
    if (int rc = validate_observable(q->observable, &probe)) return rc;
    if (q->gradient && !q->observable->hermitian) {
      set_error("adjoint gradients need a Hermitian observable");
      return MB_EUNSUPPORTED;
    }
    if (q->gradient) {
      for (const COp& op : b->ops)
        if (op.gen_off >= 0 && op.k > 5) {
          set_error("gradient of a gate with more than 5 positions");
          return MB_EUNSUPPORTED;
        }
    }
    Class* c = find_class(S, b, dm);
    if (!c) {
      if (int rc = make_class(S, b, dm, &c)) return rc;
    }
    r->cls = c;
    r->obs = q->observable;
    r->gradient = q->gradient ? 1 : 0;
    r->L = q->repeats;
    r->theta.assign(q->theta, q->theta + nt);
  }
  std::lock_guard<std::mutex> lk(S->qmu);
  if (S->stop) {
    set_error("the server is stopping");
    return MB_EINVAL;
  }
  r->ticket = S->next_ticket++;
  r->t_submit = now_ms();
  if (S->t_first < 0) S->t_first = r->t_submit;
  *ticket = r->ticket;
  S->inflight.insert(r->ticket);
  ++S->submitted;
  ++S->n_pending;
  S->incoming.push_back(r.release());
  S->qcv.notify_one();
  return MB_OK;
}

extern "C" int mb_poll(mb_server S, uint64_t ticket, mb_result* res, double* grad, size_t ngrad) {
  if (!S) return MB_EINVAL;
  std::lock_guard<std::mutex> lk(S->qmu);
  auto it = S->finished.find(ticket);
  if (it == S->finished.end()) {
    if (S->inflight.count(ticket)) return MB_ENOTREADY;
    set_error("unknown ticket %llu", (unsigned long long)ticket);
    return MB_EINVAL;
  }
  if (int rc = copy_result(it->second, res, grad, ngrad)) return rc;
  delete it->second;
  S->finished.erase(it);
  return MB_OK;
}

extern "C" int mb_wait(mb_server S, uint64_t ticket, int timeout_ms, mb_result* res, double* grad, size_t ngrad) {
  if (!S) return MB_EINVAL;
  std::unique_lock<std::mutex> lk(S->qmu);
  auto ready = [&] { return S->finished.count(ticket) || !S->inflight.count(ticket); };
  if (timeout_ms < 0) S->done_cv.wait(lk, ready);
  else if (!S->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return MB_ETIMEOUT;
  auto it = S->finished.find(ticket);
  if (it == S->finished.end()) {
    set_error("unknown ticket %llu", (unsigned long long)ticket);
    return MB_EINVAL;
  }
  if (int rc = copy_result(it->second, res, grad, ngrad)) return rc;
  delete it->second;
  S->finished.erase(it);
  return MB_OK;
}

extern "C" int mb_server_stats_get(mb_server S, mb_server_stats* o) {
  if (!S || !o) return MB_EINVAL;
  std::lock_guard<std::mutex> lk(S->qmu);
  std::memset(o, 0, sizeof(*o));
  o->submitted = S->submitted;
  o->completed = S->completed;
  o->failed = S->failed;
  o->iterations = S->iterations;
  o->active = S->n_active;
  o->pending = S->n_pending;
  o->bytes_in_use = S->used;
  o->peak_bytes = S->peak;
  o->budget_bytes = S->budget;
  if (!S->lat.empty()) {
    std::vector<double> v = S->lat;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
      const double pos = q * double(v.size() - 1);
      const size_t i = size_t(pos);
      const double f = pos - double(i);
      return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
    };
    o->p50_ms = pct(0.50);
    o->p99_ms = pct(0.99);
    const double span = S->t_last - S->t_first;
    o->evals_per_s = span > 0 ? double(S->completed) / (span / 1e3) : 0.0;
  }
  double ms = 0;
  uint64_t nc = 0;
  jit_stats(&ms, &nc, nullptr);
  o->jit_compile_ms = ms - S->jit_ms0;
  o->jit_compiles = nc - S->jit_n0;
  return MB_OK;
}

extern "C" int mb_server_stats_reset(mb_server S) {
  if (!S) return MB_EINVAL;
  std::lock_guard<std::mutex> lk(S->qmu);
  S->lat.clear();
  S->submitted = S->completed = S->failed = S->iterations = 0;
  S->t_first = -1;
  jit_stats(&S->jit_ms0, &S->jit_n0, nullptr);
  S->t_last = 0;
  S->peak = S->used;
  return MB_OK;
}

extern "C" int mb_server_stop(mb_server S) {
  if (!S) return MB_OK;
  {
    std::lock_guard<std::mutex> lk(S->qmu);
    S->stop = true;
  }
  S->qcv.notify_all();
  if (S->th.joinable()) S->th.join();
  std::lock_guard<std::recursive_mutex> g(g_mu);
  if (g_ctx.init) {
    cudaStreamSynchronize(g_ctx.stream);
    for (auto& c : S->classes) {
      dev_free(c->pool);
      dev_free(c->d_theta);
      circuit_release(c->priv);
    }
    dev_free(S->d_res);
  }
  S->classes.clear();
  for (auto& kv : S->finished) delete kv.second;
  for (Req* r : S->incoming) delete r;
  if (S->arena) cudaFreeHost(S->arena);
  if (S->ev) cudaEventDestroy(S->ev);
  --g_servers_running;
  delete S;
  return MB_OK;
}

namespace mb {
int servers_running() { return g_servers_running; }
}  // namespace mb
