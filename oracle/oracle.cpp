// CPU oracle: a C++ restatement of MOSSQuantum's dense ComplexF64 CPU simulator.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA backend in
// mossquantum_b200/. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg may load it. The product path never calls it.
//
// Every routine cites the reference file it restates (paths inside MOSSQuantum):
//   gate sweep ............ src/backends/cpu/gates/serial_short_range.jl:2-71,
//                           src/backends/cpu/gates/threaded_long_range.jl:3-132
//   CNOT / CZ ............. src/backends/cpu/gates/specific/cz_gate.jl:1-71
//   density two-pass ...... src/backends/cpu/gates/generic.jl:24-34
//   channel supermatrix ... src/backends/cpu/gates/channels.jl:2-35,
//                           src/quantum_circuits/channels/quantum_map.jl:59-67
//   expectation ........... src/observables/expectation.jl:12-73,
//                           src/observables/density_matrix_expectation.jl:1-25
//   probabilities ......... src/execution/probabilities.jl:8-105
//   adjoint ............... src/differentiation/circuit.jl:77-229,
//                           src/differentiation/expectation.jl:4-73
//   threading ............. src/utils/parallel_for.jl:3-80
//
// Complex numbers are stored interleaved (re, im) like Julia's ComplexF64, matrices
// column-major like Julia's Matrix. Positions are zero-based bit indices (reference
// position q is bit q-1). Every matrix handed in is already in "ordered" form
// (ordered_mat / ordered_supermat): positions ascending, first position = least
// significant local bit.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct cplx {
  double re, im;
};
static inline cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static inline cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
static inline cplx cconj(cplx a) { return {a.re, -a.im}; }

// Minimum work per task (src/utils/parallel_for.jl:3-6).
constexpr int64_t kMinSize = 1024;
constexpr int64_t kDenseGateMinWork = 256;
constexpr int64_t kSwapMinWork = 16384;
constexpr int64_t kPhaseMinWork = 32768;

int g_threads = 1;

// Persistent worker pool behind parallel_run / parallel_sum: the reference schedules its
// ranges as tasks on Julia's resident thread pool, so threads are started once here too
// rather than once per gate. The calling thread runs task 0 itself.
class Pool {
 public:
  ~Pool() { resize(0); }
  // Runs f(p) for p = 0..tasks-1 and returns when all have finished.
  void run(int64_t tasks, const std::function<void(int64_t)>& f) {
    if (tasks <= 1) {
      if (tasks == 1) f(0);
      return;
    }
    std::lock_guard<std::mutex> serial(run_mu_);
    if (int64_t(workers_.size()) < tasks - 1) resize(int(tasks - 1));
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &f;
      tasks_ = tasks;
      next_ = 1;          // task 0 runs on the calling thread
      pending_ = tasks - 1;
      ++gen_;
    }
    cv_.notify_all();
    f(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
    tasks_ = 0;
  }

 private:
  void resize(int n) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
    workers_.clear();
    stop_ = false;
    for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
  }
  // A task index and the job it belongs to are taken in one critical section, so a worker that
  // wakes late can never pair a finished job with the next job's counter.
  void loop() {
    std::unique_lock<std::mutex> lk(mu_);
    uint64_t seen = gen_;
    for (;;) {
      cv_.wait(lk, [&] { return gen_ != seen || (job_ && next_ < tasks_); });
      seen = gen_;
      if (stop_) return;
      while (job_ && next_ < tasks_) {
        const int64_t p = next_++;
        const std::function<void(int64_t)>* job = job_;
        lk.unlock();
        (*job)(p);
        lk.lock();
        if (--pending_ == 0) done_cv_.notify_one();
      }
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, run_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int64_t)>* job_ = nullptr;
  int64_t tasks_ = 0, pending_ = 0, next_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

Pool& pool() {
  static Pool p;
  return p;
}

// parallel_run (src/utils/parallel_for.jl:9-45): contiguous zero-based inclusive ranges
// [total*p/tasks, total*(p+1)/tasks - 1], tasks = max(1, min(threads, total / min_work)).
void parallel_run(int64_t total, int64_t min_work, const std::function<void(int64_t, int64_t)>& f) {
  int64_t tasks = std::max<int64_t>(1, std::min<int64_t>(g_threads, total / min_work));
  if (tasks == 1) {
    if (total > 0) f(0, total - 1);
    return;
  }
  pool().run(tasks, [&](int64_t p) {
    const int64_t ist = total * p / tasks, ifn = total * (p + 1) / tasks - 1;
    if (ifn >= ist) f(ist, ifn);
  });
}

// parallel_sum (src/utils/parallel_for.jl:47-80): partitions into n_threads ranges when
// total >= MIN_SIZE and sums the partial results.
cplx parallel_sum(int64_t total, const std::function<cplx(int64_t, int64_t)>& f) {
  if (total >= kMinSize && g_threads > 1) {
    const int tasks = g_threads;
    std::vector<cplx> part(tasks, cplx{0, 0});
    pool().run(tasks, [&](int64_t p) {
      const int64_t ist = total * p / tasks, ifn = total * (p + 1) / tasks - 1;
      part[p] = ifn >= ist ? f(ist, ifn) : cplx{0, 0};
    });
    cplx r{0, 0};
    for (auto& v : part) r = cadd(r, v);
    return r;
  }
  return total > 0 ? f(0, total - 1) : cplx{0, 0};
}

// Insert zero bits at the (ascending) positions pos[0..k-1] into the compact index i.
static inline int64_t insert_zeros(int64_t i, int k, const int* pos) {
  for (int j = 0; j < k; ++j) {
    int64_t low = i & ((int64_t(1) << pos[j]) - 1);
    i = ((i >> pos[j]) << (pos[j] + 1)) | low;
  }
  return i;
}

// Small k with the block size known at compile time; the arithmetic (and its order) is the
// generic loop's, so results are identical.
template <int K>
void apply_dense_k(cplx* v, int64_t len, const int* pos, const cplx* m) {
  constexpr int d = 1 << K;
  int64_t off[d];
  for (int a = 0; a < d; ++a) {
    int64_t o = 0;
    for (int j = 0; j < K; ++j)
      if ((a >> j) & 1) o |= int64_t(1) << pos[j];
    off[a] = o;
  }
  parallel_run(len >> K, kDenseGateMinWork, [&](int64_t ist, int64_t ifn) {
    cplx in[d], out[d];
    for (int64_t b = ist; b <= ifn; ++b) {
      const int64_t base = insert_zeros(b, K, pos);
      for (int a = 0; a < d; ++a) in[a] = v[base + off[a]];
      for (int r = 0; r < d; ++r) {
        cplx acc = cmul(m[r], in[0]);
        for (int c = 1; c < d; ++c) acc = cadd(acc, cmul(m[r + c * d], in[c]));
        out[r] = acc;
      }
      for (int a = 0; a < d; ++a) v[base + off[a]] = out[a];
    }
  });
}

// Generic k-qubit sweep (k <= 10 so channels on up to 5 qubits fit): for every block of
// 2^k amplitudes sharing the other bits, v_local <- M v_local, local bit j = bit pos[j].
// Restates _apply_gate_2_impl! (serial_short_range.jl:2-71) and the 4/5-body kernels
// (threaded_long_range.jl:3-132); the sum over j runs in ascending order like the
// StaticArrays product M * v.
void apply_dense(cplx* v, int64_t len, int k, const int* pos, const cplx* m) {
  if (k == 1) return apply_dense_k<1>(v, len, pos, m);
  if (k == 2) return apply_dense_k<2>(v, len, pos, m);
  if (k == 3) return apply_dense_k<3>(v, len, pos, m);
  const int d = 1 << k;
  std::vector<int64_t> off(d);
  for (int a = 0; a < d; ++a) {
    int64_t o = 0;
    for (int j = 0; j < k; ++j)
      if ((a >> j) & 1) o |= int64_t(1) << pos[j];
    off[a] = o;
  }
  int64_t blocks = len >> k;
  parallel_run(blocks, kDenseGateMinWork, [&](int64_t ist, int64_t ifn) {
    std::vector<cplx> in(d), out(d);
    for (int64_t b = ist; b <= ifn; ++b) {
      int64_t base = insert_zeros(b, k, pos);
      for (int a = 0; a < d; ++a) in[a] = v[base + off[a]];
      for (int r = 0; r < d; ++r) {
        cplx acc = cmul(m[r], in[0]);
        for (int c = 1; c < d; ++c) acc = cadd(acc, cmul(m[r + c * d], in[c]));
        out[r] = acc;
      }
      for (int a = 0; a < d; ++a) v[base + off[a]] = out[a];
    }
  });
}

// CNOT (cz_gate.jl:27-71): swap the target pair where the control bit is set.
void apply_cnot(cplx* v, int64_t len, int control, int target) {
  int q[2] = {std::min(control, target), std::max(control, target)};
  int64_t pc = int64_t(1) << control, pt = int64_t(1) << target;
  parallel_run(len >> 2, kSwapMinWork, [&](int64_t ist, int64_t ifn) {
    for (int64_t i = ist; i <= ifn; ++i) {
      int64_t l00 = insert_zeros(i, 2, q);
      std::swap(v[l00 | pc], v[l00 | pc | pt]);
    }
  });
}

// CZ (cz_gate.jl:1-25): negate the amplitudes with both bits set.
void apply_cz(cplx* v, int64_t len, int a, int b) {
  int q[2] = {std::min(a, b), std::max(a, b)};
  int64_t mask = (int64_t(1) << a) | (int64_t(1) << b);
  parallel_run(len >> 2, kPhaseMinWork, [&](int64_t ist, int64_t ifn) {
    for (int64_t i = ist; i <= ifn; ++i) {
      int64_t l = insert_zeros(i, 2, q) | mask;
      v[l] = {-v[l].re, -v[l].im};
    }
  });
}

enum { OP_GATE = 0, OP_CHANNEL = 1, OP_CNOT = 2, OP_CZ = 3 };

}  // namespace

extern "C" {

// One instruction of a bound circuit.
//  kind  OP_GATE: unitary gate, mat = ordered_mat (2^nq x 2^nq)
//        OP_CHANNEL: mat = ordered_supermat (4^nq x 4^nq), valid on density matrices
//        OP_CNOT: pos[0] = control, pos[1] = target (given order, not sorted)
//        OP_CZ: pos[0], pos[1]
//  gens  nparams derivative generators D = (dU)'U in ordered form (same shape as mat)
typedef struct or_op {
  int32_t kind;
  int32_t nq;
  int32_t pos[5];
  int32_t nparams;
  const double* mat;
  const double* gens;
} or_op;

// One observable key: sorted sites, dense local matrix (2^k x 2^k) = the sum of that
// key's terms (src/backends/cpu/operators/utils.jl:8-20).
typedef struct or_key {
  int32_t k;
  int32_t pos[5];
  const double* mat;
} or_key;

void or_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int or_get_threads(void) { return g_threads; }

static void conj_transpose(const cplx* m, int d, std::vector<cplx>& out) {
  out.resize(size_t(d) * d);
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c) out[c + r * d] = cconj(m[r + c * d]);
}

// Apply one op. is_dm: state is a vectorised 2^n x 2^n column-major density matrix.
// dagger: apply the adjoint (U' for gates, S' for channels; apply_dagger!).
static void apply_op(const or_op& op, cplx* v, int n, int is_dm, int dagger) {
  int64_t len = is_dm ? (int64_t(1) << (2 * n)) : (int64_t(1) << n);
  const cplx* m = reinterpret_cast<const cplx*>(op.mat);
  if (op.kind == OP_CNOT) {
    apply_cnot(v, len, op.pos[0], op.pos[1]);
    if (is_dm) apply_cnot(v, len, op.pos[0] + n, op.pos[1] + n);
    return;
  }
  if (op.kind == OP_CZ) {
    apply_cz(v, len, op.pos[0], op.pos[1]);
    if (is_dm) apply_cz(v, len, op.pos[0] + n, op.pos[1] + n);
    return;
  }
  if (op.kind == OP_CHANNEL) {
    // _qmap_apply_threaded! (channels.jl:2-24): supermatrix on (pos..., pos+n...).
    int k = 2 * op.nq;
    int pos[10];
    for (int j = 0; j < op.nq; ++j) { pos[j] = op.pos[j]; pos[j + op.nq] = op.pos[j] + n; }
    int d = 1 << k;
    if (dagger) {
      std::vector<cplx> md;
      conj_transpose(m, d, md);
      apply_dense(v, len, k, pos, md.data());
    } else {
      apply_dense(v, len, k, pos, m);
    }
    return;
  }
  int k = op.nq;
  int d = 1 << k;
  std::vector<cplx> mm(m, m + size_t(d) * d);
  if (dagger) conj_transpose(m, d, mm);
  if (k == 0) {
    // Zero-qubit gate: scalar multiple (generic.jl:1-9).
    for (int64_t i = 0; i < len; ++i) v[i] = cmul(mm[0], v[i]);
    if (is_dm) for (int64_t i = 0; i < len; ++i) v[i] = cmul(cconj(mm[0]), v[i]);
    return;
  }
  apply_dense(v, len, k, op.pos, mm.data());
  if (is_dm) {
    // _dm_apply_threaded! (generic.jl:24-34): conj(U) on the column bits pos+n.
    int pos2[5];
    for (int j = 0; j < k; ++j) pos2[j] = op.pos[j] + n;
    for (auto& x : mm) x = cconj(x);
    apply_dense(v, len, k, pos2, mm.data());
  }
}

// Apply a bound circuit in order (execution/gates.jl:21-36).
int or_apply_circuit(const or_op* ops, int nops, double* state, int n, int is_dm) {
  cplx* v = reinterpret_cast<cplx*>(state);
  for (int i = 0; i < nops; ++i) {
    if (ops[i].kind == OP_CHANNEL && !is_dm) return -1;
    apply_op(ops[i], v, n, is_dm, 0);
  }
  return 0;
}

// Apply a single dense matrix on explicit positions (used to build test cases).
void or_apply_matrix(double* state, int64_t len, int k, const int* pos, const double* mat) {
  apply_dense(reinterpret_cast<cplx*>(state), len, k, pos, reinterpret_cast<const cplx*>(mat));
}

// <c| M_key |v> summed over keys, M acting on the key's sites
// (expectation_value threaded kernels, src/backends/cpu/expectations/threaded*.jl).
static cplx cross_keys(const cplx* c, const cplx* v, int n, const or_key* keys, int nkeys) {
  int64_t len = int64_t(1) << n;
  cplx total{0, 0};
  for (int q = 0; q < nkeys; ++q) {
    const or_key& key = keys[q];
    const cplx* m = reinterpret_cast<const cplx*>(key.mat);
    int k = key.k, d = 1 << k;
    if (k == 0) {
      cplx dot = parallel_sum(len, [&](int64_t ist, int64_t ifn) {
        cplx acc{0, 0};
        for (int64_t i = ist; i <= ifn; ++i) acc = cadd(acc, cmul(cconj(c[i]), v[i]));
        return acc;
      });
      total = cadd(total, cmul(m[0], dot));
      continue;
    }
    std::vector<int64_t> off(d);
    for (int a = 0; a < d; ++a) {
      int64_t o = 0;
      for (int j = 0; j < k; ++j) if ((a >> j) & 1) o |= int64_t(1) << key.pos[j];
      off[a] = o;
    }
    cplx r = parallel_sum(len >> k, [&](int64_t ist, int64_t ifn) {
      cplx acc{0, 0};
      for (int64_t b = ist; b <= ifn; ++b) {
        int64_t base = insert_zeros(b, k, key.pos);
        for (int row = 0; row < d; ++row) {
          cplx mv{0, 0};
          for (int col = 0; col < d; ++col) mv = cadd(mv, cmul(m[row + col * d], v[base + off[col]]));
          acc = cadd(acc, cmul(cconj(c[base + off[row]]), mv));
        }
      }
      return acc;
    });
    total = cadd(total, r);
  }
  return total;
}

// tr(M rho) summed over keys (density_matrix_expectation.jl:1-25):
// sum_base sum_{a,b} M[a,b] rho[base|b, base|a].
static cplx trace_keys(const cplx* rho, int n, const or_key* keys, int nkeys) {
  int64_t dim = int64_t(1) << n;
  cplx total{0, 0};
  for (int q = 0; q < nkeys; ++q) {
    const or_key& key = keys[q];
    const cplx* m = reinterpret_cast<const cplx*>(key.mat);
    int k = key.k, d = 1 << k;
    std::vector<int64_t> off(d);
    for (int a = 0; a < d; ++a) {
      int64_t o = 0;
      for (int j = 0; j < k; ++j) if ((a >> j) & 1) o |= int64_t(1) << key.pos[j];
      off[a] = o;
    }
    cplx r{0, 0};
    for (int64_t b = 0; b < (dim >> k); ++b) {
      int64_t base = insert_zeros(b, k, key.pos);
      for (int a = 0; a < d; ++a)
        for (int bb = 0; bb < d; ++bb) {
          int64_t row = base + off[bb], col = base + off[a];
          r = cadd(r, cmul(m[a + bb * d], rho[row + col * dim]));
        }
    }
    total = cadd(total, r);
  }
  return total;
}

// Expectation of an observable (sum of keys). out = complex (re, im).
int or_expect(const double* state, int n, int is_dm, const or_key* keys, int nkeys, double* out) {
  const cplx* v = reinterpret_cast<const cplx*>(state);
  cplx r = is_dm ? trace_keys(v, n, keys, nkeys) : cross_keys(v, v, n, keys, nkeys);
  out[0] = r.re;
  out[1] = r.im;
  return 0;
}

// <c|H|v> (observables/expectation.jl:59-73).
int or_cross_expect(const double* cstate, const double* state, int n, const or_key* keys, int nkeys, double* out) {
  cplx r = cross_keys(reinterpret_cast<const cplx*>(cstate), reinterpret_cast<const cplx*>(state), n, keys, nkeys);
  out[0] = r.re;
  out[1] = r.im;
  return 0;
}

// out = sum_keys M_key v (observable action, execution/operators.jl:41-57). For a
// density matrix (is_dm) the action is on the row bits: out = H * rho.
int or_apply_observable(const double* state, double* outp, int n, int is_dm, const or_key* keys, int nkeys) {
  int64_t len = is_dm ? (int64_t(1) << (2 * n)) : (int64_t(1) << n);
  const cplx* v = reinterpret_cast<const cplx*>(state);
  cplx* out = reinterpret_cast<cplx*>(outp);
  std::fill(out, out + len, cplx{0, 0});
  std::vector<cplx> tmp(len);
  for (int q = 0; q < nkeys; ++q) {
    std::copy(v, v + len, tmp.begin());
    if (keys[q].k == 0) {
      cplx s = reinterpret_cast<const cplx*>(keys[q].mat)[0];
      for (int64_t i = 0; i < len; ++i) out[i] = cadd(out[i], cmul(s, tmp[i]));
      continue;
    }
    apply_dense(tmp.data(), len, keys[q].k, keys[q].pos, reinterpret_cast<const cplx*>(keys[q].mat));
    for (int64_t i = 0; i < len; ++i) out[i] = cadd(out[i], tmp[i]);
  }
  return 0;
}

// Marginal probabilities (probabilities.jl:42-84). qubits: zero-based, the first one is
// the least significant bit of the output index. Returns -2 when the state is not
// normalised within sqrt(eps), -3 on a negative entry beyond tolerance.
int or_probabilities(const double* state, int n, int is_dm, const int* qubits, int nq, double* out) {
  const cplx* v = reinterpret_cast<const cplx*>(state);
  int64_t dim = int64_t(1) << n;
  int64_t m = int64_t(1) << nq;
  std::fill(out, out + m, 0.0);
  double tol = std::sqrt(2.220446049250313e-16);
  for (int64_t i = 0; i < dim; ++i) {
    int64_t idx = 0;
    for (int j = 0; j < nq; ++j) idx |= ((i >> qubits[j]) & 1) << j;
    double p;
    if (is_dm) {
      cplx x = v[i + i * dim];
      if (std::fabs(x.im) > tol) return -4;
      p = x.re;
    } else {
      p = v[i].re * v[i].re + v[i].im * v[i].im;
    }
    out[idx] += p;
  }
  double mn = out[0], total = 0;
  for (int64_t i = 0; i < m; ++i) mn = std::min(mn, out[i]);
  if (mn < -tol) return -3;
  for (int64_t i = 0; i < m; ++i) { out[i] = std::max(out[i], 0.0); total += out[i]; }
  if (!(std::fabs(total - 1) <= std::max(tol, tol * std::max(std::fabs(total), 1.0)))) return -2;
  for (int64_t i = 0; i < m; ++i) out[i] /= total;
  return 0;
}

// Adjoint gradient of Re<H> (differentiation/circuit.jl:77-229, expectation.jl:4-73,
// objectives.jl:183-213) with seed 1.
//  state0: initial state (pure 2^n or density 4^n entries, by is_dm).
//  The observable must be Hermitian (the reference's support check).
//  grads: one entry per active parameter, forward circuit order.
//  Pure initial states followed by channels are promoted to density matrices at the
//  first channel and the cotangent is mapped back with (D + D')x (circuit.jl:62-66).
int or_adjoint(const or_op* ops, int nops, const double* state0, int n, int is_dm, const or_key* keys,
               int nkeys, double* value, double* grads) {
  int64_t dimp = int64_t(1) << n, dimd = int64_t(1) << (2 * n);
  // Forward with checkpoints of channel inputs.
  bool has_channel = false;
  for (int i = 0; i < nops; ++i) has_channel |= ops[i].kind == OP_CHANNEL;
  std::vector<cplx> y(is_dm ? dimd : dimp);
  std::memcpy(y.data(), state0, y.size() * sizeof(cplx));
  bool dm = is_dm;
  std::vector<std::vector<cplx>> ckpt(nops);
  std::vector<char> ckpt_dm(nops, 0);
  for (int i = 0; i < nops; ++i) {
    if (ops[i].kind == OP_CHANNEL) {
      ckpt[i] = y;
      ckpt_dm[i] = dm;
      if (!dm) {
        // StateVector -> DensityMatrix(psi psi') (execution/channels.jl:19).
        std::vector<cplx> rho(dimd);
        for (int64_t c = 0; c < dimp; ++c)
          for (int64_t r = 0; r < dimp; ++r) rho[r + c * dimp] = cmul(y[r], cconj(y[c]));
        y.swap(rho);
        dm = true;
      }
    }
    apply_op(ops[i], y.data(), n, dm, 0);
  }
  (void)has_channel;
  // Observation and seed.
  std::vector<cplx> delta(y.size());
  if (dm) {
    cplx e = trace_keys(y.data(), n, keys, nkeys);
    *value = e.re;
    // Seed z H' applied to the identity (expectation.jl:69-73): the dense matrix H.
    std::vector<cplx> ident(dimd, cplx{0, 0});
    for (int64_t i = 0; i < dimp; ++i) ident[i + i * dimp] = {1, 0};
    or_apply_observable(reinterpret_cast<double*>(ident.data()), reinterpret_cast<double*>(delta.data()), n, 1,
                        keys, nkeys);
  } else {
    cplx e = cross_keys(y.data(), y.data(), n, keys, nkeys);
    *value = e.re;
    // Seed (conj z) H psi + z H' psi = 2 H psi for Hermitian H (expectation.jl:32-35).
    or_apply_observable(reinterpret_cast<double*>(y.data()), reinterpret_cast<double*>(delta.data()), n, 0, keys,
                        nkeys);
    for (auto& x : delta) x = {2 * x.re, 2 * x.im};
  }
  // Reverse sweep.
  std::vector<std::vector<double>> per_gate;
  std::vector<cplx> left, right;
  for (int i = nops - 1; i >= 0; --i) {
    const or_op& op = ops[i];
    if (op.kind == OP_CHANNEL) {
      apply_op(op, delta.data(), n, 1, 1);
      y = ckpt[i];
      if (!ckpt_dm[i]) {
        // _density_to_state_cotangent: (D + D') x.
        std::vector<cplx> g(dimp, cplx{0, 0});
        for (int64_t r = 0; r < dimp; ++r) {
          cplx acc{0, 0};
          for (int64_t c = 0; c < dimp; ++c) {
            cplx dd = cadd(delta[r + c * dimp], cconj(delta[c + r * dimp]));
            acc = cadd(acc, cmul(dd, y[c]));
          }
          g[r] = acc;
        }
        delta.swap(g);
        dm = false;
      }
      continue;
    }
    apply_op(op, delta.data(), n, dm, 1);
    apply_op(op, y.data(), n, dm, 1);
    if (op.nparams > 0) {
      std::vector<double> g(op.nparams);
      int k = op.nq, d = 1 << k;
      for (int p = 0; p < op.nparams; ++p) {
        const cplx* dmat = reinterpret_cast<const cplx*>(op.gens) + size_t(p) * d * d;
        if (!dm) {
          // Re <y| D |delta> (back_propagate, circuit.jl:136-144).
          or_key key;
          key.k = k;
          for (int j = 0; j < k; ++j) key.pos[j] = op.pos[j];
          key.mat = reinterpret_cast<const double*>(dmat);
          cplx r = cross_keys(y.data(), delta.data(), n, &key, 1);
          g[p] = r.re;
        } else {
          // _density_gate_gradient! (circuit.jl:155-172): D' on rows, D^T on columns.
          left = y;
          right = y;
          std::vector<cplx> dd, dt(size_t(d) * d);
          conj_transpose(dmat, d, dd);
          for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) dt[c + r * d] = dmat[r + c * d];
          int pos2[5];
          for (int j = 0; j < k; ++j) pos2[j] = op.pos[j] + n;
          apply_dense(left.data(), dimd, k, op.pos, dd.data());
          apply_dense(right.data(), dimd, k, pos2, dt.data());
          double acc = 0;
          for (int64_t e = 0; e < dimd; ++e) {
            cplx a = cmul(cconj(delta[e]), left[e]);
            cplx b = cmul(cconj(delta[e]), right[e]);
            acc += a.re + b.re;
          }
          g[p] = acc;
        }
      }
      per_gate.push_back(g);
    }
  }
  // _flatten_gradients: forward order.
  size_t w = 0;
  for (auto it = per_gate.rbegin(); it != per_gate.rend(); ++it)
    for (double x : *it) grads[w++] = x;
  return int(w);
}

}  // extern "C"
