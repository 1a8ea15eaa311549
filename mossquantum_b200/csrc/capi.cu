// C ABI of libmossb200: context, states, circuits, observables and the host-side
// orchestration of the device kernels. See include/mossb200.h for the contract.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "internal.h"

namespace mb {

// ---------------------------------------------------------------------------------------------
// Errors and launch accounting
// ---------------------------------------------------------------------------------------------
static thread_local std::string t_error;
void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_error = buf;
}
uint64_t& launch_counter() {
  static uint64_t c = 0;
  return c;
}

Ctx g_ctx;
std::recursive_mutex g_mu;

// ---------------------------------------------------------------------------------------------
// Budgeted device allocation (stream-ordered; the pool keeps freed blocks for reuse).
// ---------------------------------------------------------------------------------------------
int dev_alloc(void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 256;
  bytes = (bytes + 255) & ~size_t(255);
  if (g_ctx.used + bytes > g_ctx.budget) {
    set_error("HBM budget exceeded: %zu bytes requested, %zu of %zu in use", bytes, g_ctx.used, g_ctx.budget);
    return MB_ENOMEM_BUDGET;
  }
  cudaError_t e = cudaMallocAsync(p, bytes, g_ctx.stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return MB_ENOMEM_BUDGET;
  }
  g_ctx.used += bytes;
  g_ctx.sizes[*p] = bytes;
  return MB_OK;
}

void dev_free(void* p) {
  if (!p) return;
  auto it = g_ctx.sizes.find(p);
  if (it != g_ctx.sizes.end()) {
    g_ctx.used -= it->second;
    g_ctx.sizes.erase(it);
  }
  cudaFreeAsync(p, g_ctx.stream);
}

int check_init() {
  if (!g_ctx.init) {
    set_error("mb_init has not been called");
    return MB_ENOTINIT;
  }
  return MB_OK;
}

ReduceWs ws() { return ReduceWs{g_ctx.partials, g_ctx.counters, g_ctx.partials_cap, g_ctx.ncounters}; }

int launch_dense_block(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* m, int64_t mstride,
                       int mode, bool allow_tensor, cudaStream_t st) {
  static const bool disabled = getenv("MB_DMMA") && atoi(getenv("MB_DMMA")) == 0;
  if (allow_tensor && !disabled && mstride == 0 && (pos.k == 4 || pos.k == 5)) {
    const int rc = launch_dmma(v, elems, nsamples, pos, m, mode, st);
    if (rc != MB_EUNSUPPORTED) return rc;
  }
  return launch_dense(v, elems, nsamples, pos, m, mstride, mode, st);
}

// ---------------------------------------------------------------------------------------------
// Small host helpers
// ---------------------------------------------------------------------------------------------
typedef std::complex<double> cd;

static bool finite_mat(const double* m, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(m[i])) return false;
  return true;
}

// ordered local index a' -> own-order local index (gates/abstract_gates.jl:162-166)
static void norm_order(int k, const int* pos, int* sorted_pos, int* perm) {
  int seq[5];
  for (int j = 0; j < k; ++j) seq[j] = j;
  std::sort(seq, seq + k, [&](int a, int b) { return pos[a] < pos[b]; });
  for (int j = 0; j < k; ++j) sorted_pos[j] = pos[seq[j]];
  for (int ap = 0; ap < (1 << k); ++ap) {
    int a = 0;
    for (int j = 0; j < k; ++j)
      if ((ap >> j) & 1) a |= 1 << seq[j];
    perm[ap] = a;
  }
}

static int family_arity(int fam) {
  switch (fam) {
    case MB_FAM_RX: case MB_FAM_RY: case MB_FAM_RZ: case MB_FAM_PHASE: return 1;
    case MB_FAM_CRX: case MB_FAM_CRY: case MB_FAM_CRZ: case MB_FAM_CPHASE: return 2;
    case MB_FAM_CCPHASE: return 3;
    case MB_FAM_SELECT: return 0;  // 1..3 positions, checked separately
    default: return -1;
  }
}

static double2 d2(cd x) { return make_double2(x.real(), x.imag()); }

}  // namespace mb

using namespace mb;

// =============================================================================================
// Context
// =============================================================================================
extern "C" int mb_init(int device, size_t hbm_budget_bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (g_ctx.init) {
    if (device != g_ctx.device) {
      set_error("already initialised on device %d", g_ctx.device);
      return MB_EINVAL;
    }
    if (hbm_budget_bytes) g_ctx.budget = hbm_budget_bytes;
    return MB_OK;
  }
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error("no CUDA device available (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    return MB_EDEVICE;
  }
  if (device < 0 || device >= count) {
    set_error("device %d out of range (0..%d)", device, count - 1);
    return MB_EINVAL;
  }
  MB_CHECK_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  MB_CHECK_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    set_error("device %d (%s, sm_%d%d) is not a Blackwell sm_100 GPU", device, prop.name, prop.major, prop.minor);
    return MB_EUNSUPPORTED;
  }
  g_ctx.device = device;
  g_ctx.sm_count = prop.multiProcessorCount;
  MB_CHECK_CUDA(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
  cudaMemPool_t pool;
  MB_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t thresh = UINT64_MAX;
  MB_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
  size_t free_b = 0, total_b = 0;
  MB_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
  g_ctx.budget = hbm_budget_bytes ? hbm_budget_bytes : size_t(double(free_b) * 0.9);
  g_ctx.used = 0;
  g_ctx.init = true;
  // Reduction workspace and small result buffers.
  g_ctx.partials_cap = int64_t(1) << 16;
  g_ctx.ncounters = 8192;
  int rc;
  if ((rc = dev_alloc((void**)&g_ctx.partials, sizeof(double2) * g_ctx.partials_cap)) ||
      (rc = dev_alloc((void**)&g_ctx.counters, sizeof(unsigned) * g_ctx.ncounters)) ||
      (rc = dev_alloc((void**)&g_ctx.results, sizeof(double2) * 65536)) ||
      (rc = dev_alloc((void**)&g_ctx.flags, sizeof(unsigned) * 8))) {
    g_ctx.init = false;
    return rc;
  }
  MB_CHECK_CUDA(cudaMemsetAsync(g_ctx.counters, 0, sizeof(unsigned) * g_ctx.ncounters, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  launch_counter() = 0;
  return MB_OK;
}

extern "C" int mb_shutdown(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g_ctx.init) return MB_OK;
  if (servers_running()) {
    set_error("stop every server (mb_server_stop) before mb_shutdown");
    return MB_EINVAL;
  }
  cudaStreamSynchronize(g_ctx.stream);
  dev_free(g_ctx.partials);
  dev_free(g_ctx.counters);
  dev_free(g_ctx.results);
  dev_free(g_ctx.flags);
  cudaStreamSynchronize(g_ctx.stream);
  cudaStreamDestroy(g_ctx.stream);
  g_ctx = Ctx();
  return MB_OK;
}

extern "C" const char* mb_last_error(void) { return t_error.c_str(); }

extern "C" int mb_memory_info(size_t* used, size_t* budget) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (used) *used = g_ctx.used;
  if (budget) *budget = g_ctx.budget;
  return MB_OK;
}

extern "C" int mb_synchronize(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_version(void) { return 10000; }

extern "C" int mb_launch_count(uint64_t* launches) {
  if (!launches) return MB_EINVAL;
  *launches = launch_counter();
  return MB_OK;
}

// =============================================================================================
// States
// =============================================================================================
namespace mb {
int state_alloc(int kind, int n, int batch, mb_state* out) {
  if (kind < MB_PURE || kind > MB_BATCH_DENSITY) {
    set_error("unknown state kind %d", kind);
    return MB_EINVAL;
  }
  bool dm = kind == MB_DENSITY || kind == MB_BATCH_DENSITY;
  if (n < 0 || n > (dm ? 15 : 32)) {
    set_error("%d qubits out of range for a %s", n, dm ? "density matrix" : "state vector");
    return MB_EINVAL;
  }
  bool is_batch = kind >= MB_BATCH_PURE;
  if (is_batch && batch < 0) {
    set_error("batch size must be nonnegative");
    return MB_EINVAL;
  }
  auto s = new mb_state_s();
  s->kind = kind;
  s->n = n;
  s->batch = is_batch ? batch : 1;
  s->dim = int64_t(1) << n;
  s->elems = dm ? s->dim * s->dim : s->dim;
  s->bytes = size_t(s->elems) * s->batch * sizeof(double2);
  if (s->bytes) {
    int rc = dev_alloc((void**)&s->d, s->bytes);
    if (rc) {
      delete s;
      return rc;
    }
  }
  *out = s;
  return MB_OK;
}
}  // namespace mb

extern "C" int mb_state_create(int kind, int n, int batch, mb_state* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_state_create")) return rc;
  if (!out) return MB_EINVAL;
  int rc = state_alloc(kind, n, batch, out);
  if (rc) return rc;
  return launch_set_basis((*out)->d, (*out)->elems, (*out)->batch, 0, g_ctx.stream);
}

extern "C" int mb_state_free(mb_state s) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!s) return MB_OK;
  if (g_ctx.init) dev_free(s->d);
  delete s;
  return MB_OK;
}

extern "C" int mb_state_set_zero(mb_state s) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!s) return MB_EINVAL;
  return launch_set_basis(s->d, s->elems, s->batch, 0, g_ctx.stream);
}

extern "C" int mb_state_upload(mb_state s, const double* host, size_t n_doubles) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_state_upload")) return rc;
  if (!s || (!host && n_doubles)) return MB_EINVAL;
  if (n_doubles != size_t(s->elems) * s->batch * 2) {
    set_error("upload of %zu doubles into a state of %zu doubles", n_doubles, size_t(s->elems) * s->batch * 2);
    return MB_EINVAL;
  }
  MB_CHECK_CUDA(cudaMemcpyAsync(s->d, host, n_doubles * sizeof(double), cudaMemcpyHostToDevice, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_state_download(mb_state s, double* host, size_t n_doubles) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_state_download")) return rc;
  if (!s || (!host && n_doubles)) return MB_EINVAL;
  if (n_doubles != size_t(s->elems) * s->batch * 2) {
    set_error("download of %zu doubles from a state of %zu doubles", n_doubles, size_t(s->elems) * s->batch * 2);
    return MB_EINVAL;
  }
  MB_CHECK_CUDA(cudaMemcpyAsync(host, s->d, n_doubles * sizeof(double), cudaMemcpyDeviceToHost, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_state_copy(mb_state dst, mb_state src) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!dst || !src) return MB_EINVAL;
  if (dst->kind != src->kind || dst->n != src->n || dst->batch != src->batch) {
    set_error("copy between states of different shape");
    return MB_EINVAL;
  }
  if (dst == src || !src->bytes) return MB_OK;
  MB_CHECK_CUDA(cudaMemcpyAsync(dst->d, src->d, src->bytes, cudaMemcpyDeviceToDevice, g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_state_info(mb_state s, int* kind, int* n, int* batch) {
  if (!s) return MB_EINVAL;
  if (kind) *kind = s->kind;
  if (n) *n = s->n;
  if (batch) *batch = s->batch;
  return MB_OK;
}

extern "C" int mb_state_device_ptr(mb_state s, void** p) {
  if (!s || !p) return MB_EINVAL;
  *p = s->d;
  return MB_OK;
}

extern "C" int mb_state_to_density(mb_state src, mb_state dst) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!src || !dst) return MB_EINVAL;
  bool ok = (src->kind == MB_PURE && dst->kind == MB_DENSITY) ||
            (src->kind == MB_BATCH_PURE && dst->kind == MB_BATCH_DENSITY);
  if (!ok || src->n != dst->n || src->batch != dst->batch) {
    set_error("to_density needs a pure source and a density destination of the same shape");
    return MB_EINVAL;
  }
  return launch_to_density(src->d, dst->d, src->n, src->batch, g_ctx.stream);
}

// =============================================================================================
// Circuits
// =============================================================================================
namespace mb {

// Host half of mb_circuit_create: ordered instructions, the matrix table of one parameter row
// (fixed matrices, channel supermatrices, room for bound parametric matrices and generators)
// and the bind records. Touches no device memory.
int circuit_compile_host(const mb_op* ops, size_t nops, int n, mb_circuit c) {
  c->n = n;
  int64_t off = 0;
  std::vector<double2> table;
  int max_slot = -1;
  for (size_t i = 0; i < nops; ++i) {
    const mb_op& o = ops[i];
    COp op{};
    op.kind = o.kind;
    op.k = o.nq;
    op.family = o.family;
    op.slot = o.slot;
    op.flags = o.flags;
    op.value = o.value;
    op.gen_off = -1;
    if (o.kind != MB_OP_GATE && o.kind != MB_OP_CHANNEL) {
      set_error("instruction %zu: unknown kind %d", i, o.kind);
      return MB_EUNSUPPORTED;
    }
    int kmax = o.kind == MB_OP_GATE ? 5 : 2, kmin = o.kind == MB_OP_GATE ? 0 : 1;
    if (o.nq < kmin || o.nq > kmax) {
      set_error("instruction %zu: %d positions not supported (only implement 5-qubit gates and 1-2 qubit channels)",
                i, o.nq);
      return MB_EUNSUPPORTED;
    }
    for (int j = 0; j < o.nq; ++j) {
      if (o.pos[j] < 0 || o.pos[j] >= n) {
        set_error("instruction %zu: position %d out of range for %d qubits", i, o.pos[j] + 1, n);
        return MB_EINVAL;
      }
      for (int q = 0; q < j; ++q)
        if (o.pos[q] == o.pos[j]) {
          set_error("instruction %zu: positions must be distinct", i);
          return MB_EINVAL;
        }
    }
    int perm[32];
    norm_order(o.nq, o.pos, op.pos, perm);
    const int d = 1 << o.nq;
    op.mat_off = int(off);
    if (o.kind == MB_OP_CHANNEL) {
      if (o.family != MB_FAM_MATRIX || o.nkraus < 1 || !o.data || !finite_mat(o.data, size_t(o.nkraus) * d * d * 2)) {
        set_error("instruction %zu: a channel needs finite Kraus matrices", i);
        return MB_EINVAL;
      }
      // Supermatrix of the ordered Kraus matrices (channels/quantum_map.jl:59-67):
      // S[(a + D c), (b + D e)] = sum_k K[a,b] conj(K[c,e]).
      const int D2 = d * d;
      std::vector<cd> S(size_t(D2) * D2, cd(0, 0));
      for (int kk = 0; kk < o.nkraus; ++kk) {
        const double* K = o.data + size_t(kk) * d * d * 2;
        auto Kord = [&](int ap, int bp) {
          int a = perm[ap], b = perm[bp];
          return cd(K[2 * (a + b * d)], K[2 * (a + b * d) + 1]);
        };
        for (int a = 0; a < d; ++a)
          for (int b = 0; b < d; ++b)
            for (int cc = 0; cc < d; ++cc)
              for (int e = 0; e < d; ++e)
                S[(a + d * cc) + size_t(D2) * (b + d * e)] += Kord(a, b) * std::conj(Kord(cc, e));
      }
      for (auto& x : S) table.push_back(d2(x));
      off += int64_t(D2) * D2;
      op.cls = CLS_DENSE;
      c->has_channel = true;
    } else if (o.family == MB_FAM_MATRIX) {
      if (!o.data || !finite_mat(o.data, size_t(d) * d * 2)) {
        set_error("instruction %zu: gate matrix must be finite", i);
        return MB_EINVAL;
      }
      std::vector<cd> M(size_t(d) * d);
      for (int ap = 0; ap < d; ++ap)
        for (int bp = 0; bp < d; ++bp) {
          int a = perm[ap], b = perm[bp];
          cd x(o.data[2 * (a + b * d)], o.data[2 * (a + b * d) + 1]);
          M[ap + bp * d] = x;
        }
      if (o.flags & MB_OPF_ADJOINT) {
        std::vector<cd> A(M.size());
        for (int r = 0; r < d; ++r)
          for (int q = 0; q < d; ++q) A[r + q * d] = std::conj(M[q + r * d]);
        M.swap(A);
      }
      // Classification: diagonal, monomial (one nonzero per column), dense.
      bool diag = true, mono = true;
      for (int q = 0; q < d; ++q) {
        int nz = 0;
        for (int r = 0; r < d; ++r)
          if (M[r + q * d] != cd(0, 0)) {
            ++nz;
            if (r != q) diag = false;
          }
        if (nz != 1) mono = false;
      }
      if (o.nq == 0) {
        op.cls = CLS_DENSE;
      } else if (diag) {
        op.cls = CLS_DIAG;
        for (int a = 0; a < d; ++a)
          if (M[a + a * d] != cd(1, 0)) op.active |= 1u << a;
      } else if (mono) {
        op.cls = CLS_MONO;
        for (int a = 0; a < d; ++a) {
          int r = 0;
          while (M[r + a * d] == cd(0, 0)) ++r;
          op.sigma[a] = (r == a && M[r + a * d] == cd(1, 0)) ? -1 : r;
          op.sigma_inv[a] = -1;
        }
        for (int a = 0; a < d; ++a)
          if (op.sigma[a] >= 0) op.sigma_inv[op.sigma[a]] = a;
      } else {
        op.cls = CLS_DENSE;
      }
      for (auto& x : M) table.push_back(d2(x));
      off += int64_t(d) * d;
    } else if (o.family == MB_FAM_SELECT) {
      // Operator j of nkraus, chosen per parameter row by k_bind; stored ordered after the
      // slot the bound matrix occupies.
      if (o.nq < 1 || o.nq > 3 || o.nkraus < 1 || !o.data || !finite_mat(o.data, size_t(o.nkraus) * d * d * 2)) {
        set_error("instruction %zu: a selection needs 1-3 positions and finite operators", i);
        return MB_EINVAL;
      }
      if (o.slot < 0 && !std::isfinite(o.value)) {
        set_error("instruction %zu: parameter must be finite", i);
        return MB_EINVAL;
      }
      op.parametric = true;
      op.cls = CLS_DENSE;
      BindRec br{};
      br.family = o.family;
      br.flags = 0;
      br.slot = o.slot;
      br.k = o.nq;
      br.value = o.value;
      br.mat_off = int(off);
      br.gen_off = -1;
      br.nopt = o.nkraus;
      for (int a = 0; a < d; ++a) br.perm[a] = perm[a];
      table.resize(table.size() + size_t(d) * d, cz());
      for (int kk = 0; kk < o.nkraus; ++kk) {
        const double* K = o.data + size_t(kk) * d * d * 2;
        for (int bp = 0; bp < d; ++bp)
          for (int ap = 0; ap < d; ++ap) {
            const int a = perm[ap], b = perm[bp];
            table.push_back(make_double2(K[2 * (a + b * d)], K[2 * (a + b * d) + 1]));
          }
      }
      off += int64_t(d) * d * (1 + o.nkraus);
      if (o.slot >= 0) max_slot = std::max(max_slot, o.slot);
      c->binds.push_back(br);
    } else {
      int ar = family_arity(o.family);
      if (ar < 0 || ar != o.nq) {
        set_error("instruction %zu: family %d needs %d positions", i, o.family, ar);
        return MB_EINVAL;
      }
      if (o.slot < 0 && !std::isfinite(o.value)) {
        set_error("instruction %zu: parameter must be finite", i);
        return MB_EINVAL;
      }
      op.parametric = true;
      BindRec br{};
      br.family = o.family;
      br.flags = o.flags;
      br.slot = o.slot;
      br.k = o.nq;
      br.value = o.value;
      br.mat_off = int(off);
      for (int a = 0; a < d; ++a) br.perm[a] = perm[a];
      table.resize(table.size() + size_t(d) * d, cz());
      off += int64_t(d) * d;
      if (o.slot >= 0) {
        br.gen_off = int(off);
        op.gen_off = int(off);
        table.resize(table.size() + size_t(d) * d, cz());
        off += int64_t(d) * d;
        max_slot = std::max(max_slot, o.slot);
      } else {
        br.gen_off = -1;
      }
      c->binds.push_back(br);
      // Structural classification of the families (diagonal ones touch only active entries).
      uint32_t own_active = 0;
      switch (o.family) {
        case MB_FAM_RZ: own_active = 0x3; break;
        case MB_FAM_PHASE: own_active = 0x2; break;
        case MB_FAM_CRZ: own_active = 0xA; break;        // control (bit 0) set
        case MB_FAM_CPHASE: own_active = 0x8; break;
        case MB_FAM_CCPHASE: own_active = 0x80; break;
        default: break;
      }
      if (own_active) {
        op.cls = CLS_DIAG;
        for (int ap = 0; ap < d; ++ap)
          if ((own_active >> perm[ap]) & 1) op.active |= 1u << ap;
      } else {
        op.cls = CLS_DENSE;
      }
    }
    c->ops.push_back(op);
  }
  c->nslots = max_slot + 1;
  c->table_elems = std::max<int64_t>(off, 1);
  c->fixed_table = table;
  c->fixed_table.resize(c->table_elems, cz());
  return MB_OK;
}

}  // namespace mb

extern "C" int mb_circuit_create(const mb_op* ops, size_t nops, int n, mb_circuit* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_circuit_create")) return rc;
  if (!out || (!ops && nops)) return MB_EINVAL;
  if (n < 0 || n > 32) {
    set_error("register size %d out of range", n);
    return MB_EINVAL;
  }
  std::unique_ptr<mb_circuit_s> c(new mb_circuit_s());
  c->uid = next_circuit_uid();
  if (int rc = circuit_compile_host(ops, nops, n, c.get())) return rc;
  int rc = dev_alloc((void**)&c->d_table, sizeof(double2) * c->table_elems);
  if (!rc && !c->binds.empty()) rc = dev_alloc((void**)&c->d_binds, sizeof(BindRec) * c->binds.size());
  if (rc) {
    circuit_release(c.release());
    return rc;
  }
  c->table_rows = 1;
  cudaError_t e = cudaMemcpyAsync(c->d_table, c->fixed_table.data(), sizeof(double2) * c->table_elems,
                                  cudaMemcpyHostToDevice, g_ctx.stream);
  if (e == cudaSuccess && !c->binds.empty())
    e = cudaMemcpyAsync(c->d_binds, c->binds.data(), sizeof(BindRec) * c->binds.size(), cudaMemcpyHostToDevice,
                        g_ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_ctx.stream);
  if (e != cudaSuccess) {
    set_error("circuit upload failed: %s", cudaGetErrorString(e));
    circuit_release(c.release());
    return MB_EDEVICE;
  }
  *out = c.release();
  return MB_OK;
}

namespace mb {

uint64_t next_circuit_uid() {
  static uint64_t next = 0;
  return ++next;
}

// Device buffers, pinned staging and schedules of a circuit, then the handle itself.
void circuit_release(mb_circuit c) {
  if (!c) return;
  if (g_ctx.init) {
    dev_free(c->d_table);
    dev_free(c->d_binds);
    dev_free(c->d_theta);
    release_schedules(c);
  }
  if (c->h_theta) cudaFreeHost(c->h_theta);
  delete c;
}

// Private copy of a compiled circuit: the same instructions and fixed matrices with its own
// matrix table, parameter buffer and schedules, so the serving loop can bind per-request
// parameters without touching the caller's handle.
int circuit_clone(mb_circuit src, mb_circuit* out) {
  mb_circuit c = new mb_circuit_s();
  c->uid = next_circuit_uid();
  c->n = src->n;
  c->ops = src->ops;
  c->nslots = src->nslots;
  c->has_channel = src->has_channel;
  c->fixed_table = src->fixed_table;
  c->table_elems = src->table_elems;
  c->binds = src->binds;
  c->table_rows = 1;
  int rc = dev_alloc((void**)&c->d_table, sizeof(double2) * c->table_elems);
  if (!rc && !c->binds.empty()) rc = dev_alloc((void**)&c->d_binds, sizeof(BindRec) * c->binds.size());
  if (rc) {
    circuit_release(c);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(c->d_table, c->fixed_table.data(), sizeof(double2) * c->table_elems,
                                  cudaMemcpyHostToDevice, g_ctx.stream);
  if (e == cudaSuccess && !c->binds.empty())
    e = cudaMemcpyAsync(c->d_binds, c->binds.data(), sizeof(BindRec) * c->binds.size(), cudaMemcpyHostToDevice,
                        g_ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g_ctx.stream);
  if (e != cudaSuccess) {
    set_error("circuit copy failed: %s", cudaGetErrorString(e));
    circuit_release(c);
    return MB_EDEVICE;
  }
  *out = c;
  return MB_OK;
}

}  // namespace mb

extern "C" int mb_circuit_free(mb_circuit c) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  circuit_release(c);
  return MB_OK;
}

extern "C" int mb_circuit_nslots(mb_circuit c, int* nslots) {
  if (!c || !nslots) return MB_EINVAL;
  *nslots = c->nslots;
  return MB_OK;
}

namespace mb {

// Uploads theta and evaluates every parametric matrix into the circuit's table.
// rows = 1 (shared parameters) or the batch size (per-sample parameters).
int check_not_capturing(const char* what) {
  if (g_ctx.capturing) {
    set_error("%s synchronises or allocates and cannot be recorded into a CUDA graph", what);
    return MB_EUNSUPPORTED;
  }
  return MB_OK;
}

// Validates theta and stages it into the circuit's device parameter buffer (asynchronously,
// through pinned memory); makes room for `rows` matrix-table rows.
int theta_stage(mb_circuit c, const double* theta, size_t ntheta, int rows) {
  if (ntheta != size_t(c->nslots) * rows) {
    set_error("expected %zu parameter values, got %zu", size_t(c->nslots) * rows, ntheta);
    return MB_EINVAL;
  }
  for (size_t i = 0; i < ntheta; ++i)
    if (!std::isfinite(theta[i])) {
      set_error("parameter values must be finite");
      return MB_EINVAL;
    }
  int rc;
  if (rows > c->table_rows) {
    double2* t = nullptr;
    if ((rc = dev_alloc((void**)&t, sizeof(double2) * c->table_elems * rows))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(t, c->fixed_table.data(), sizeof(double2) * c->table_elems,
                                  cudaMemcpyHostToDevice, g_ctx.stream));
    dev_free(c->d_table);
    c->d_table = t;
    c->table_rows = rows;
  }
  c->theta_rows = rows;
  if (c->binds.empty()) return MB_OK;
  size_t need = std::max<size_t>(ntheta, 1);
  if (need > c->theta_cap) {
    dev_free(c->d_theta);
    c->d_theta = nullptr;
    if ((rc = dev_alloc((void**)&c->d_theta, sizeof(double) * need))) return rc;
    c->theta_cap = need;
  }
  if (ntheta) {
    if (c->h_theta_cap < ntheta) {
      if (c->h_theta) cudaFreeHost(c->h_theta);
      MB_CHECK_CUDA(cudaMallocHost((void**)&c->h_theta, sizeof(double) * ntheta));
      c->h_theta_cap = ntheta;
    }
    MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
    std::memcpy(c->h_theta, theta, sizeof(double) * ntheta);
    MB_CHECK_CUDA(cudaMemcpyAsync(c->d_theta, c->h_theta, sizeof(double) * ntheta, cudaMemcpyHostToDevice,
                                  g_ctx.stream));
  }
  return MB_OK;
}

// Evaluates every parametric matrix from the staged theta into the table (one launch).
int bind_launch(mb_circuit c, int rows) {
  if (c->binds.empty() || rows == 0) return MB_OK;
  return launch_bind(c->d_binds, int(c->binds.size()), c->d_theta, c->nslots, rows, c->d_table, c->table_elems,
                     g_ctx.stream);
}

int bind_circuit(mb_circuit c, const double* theta, size_t ntheta, int rows) {
  int rc = theta_stage(c, theta, ntheta, rows);
  if (rc) return rc;
  return bind_launch(c, rows);
}

// Launches one instruction with the plain per-gate kernels. dagger applies U' (S' for
// channels). mrow_stride: table stride between samples (0 = shared parameters).
int plain_op(mb_circuit c, const COp& op, double2* v, int n, int is_dm, int nsamples, int64_t mrow_stride,
             bool dagger) {
  const int64_t elems = is_dm ? (int64_t(1) << (2 * n)) : (int64_t(1) << n);
  const double2* m = c->d_table + op.mat_off;
  const int64_t ms = op.parametric ? mrow_stride : 0;
  cudaStream_t st = g_ctx.stream;
  if (op.kind == MB_OP_CHANNEL) {
    Pos p{};
    p.k = 2 * op.k;
    for (int j = 0; j < op.k; ++j) {
      p.p[j] = op.pos[j];
      p.p[j + op.k] = op.pos[j] + n;
    }
    return launch_dense_block(v, elems, nsamples, p, m, 0, dagger ? MAT_ADJOINT : MAT_PLAIN, g_ctx.tensor_plain, st);
  }
  if (op.k == 0) {
    // Zero-qubit gate: a global scalar; on a density matrix |s|^2 (U rho U').
    Pos p{};
    p.k = 1;
    p.p[0] = 0;
    std::vector<double2> h(1);
    MB_CHECK_CUDA(cudaMemcpyAsync(h.data(), m, sizeof(double2), cudaMemcpyDeviceToHost, st));
    MB_CHECK_CUDA(cudaStreamSynchronize(st));
    cd s(h[0].x, h[0].y);
    if (dagger) s = std::conj(s);
    if (is_dm) s = cd(std::norm(s), 0);
    if (s == cd(1, 0) || elems == 0) return MB_OK;
    double2* tmp = nullptr;
    int rc = dev_alloc((void**)&tmp, sizeof(double2) * 4);
    if (rc) return rc;
    double2 sm[4] = {d2(s), cz(), cz(), d2(s)};
    MB_CHECK_CUDA(cudaMemcpyAsync(tmp, sm, sizeof(sm), cudaMemcpyHostToDevice, st));
    if (n == 0) {
      // 1-element register: scale by s through the generic scale kernel (complex s).
      std::vector<double2> one(size_t(nsamples) * elems);
      MB_CHECK_CUDA(cudaMemcpyAsync(one.data(), v, sizeof(double2) * one.size(), cudaMemcpyDeviceToHost, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
      for (auto& x : one) x = d2(s * cd(x.x, x.y));
      MB_CHECK_CUDA(cudaMemcpyAsync(v, one.data(), sizeof(double2) * one.size(), cudaMemcpyHostToDevice, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
    } else {
      rc = launch_diag(v, elems, nsamples, p, tmp, 0, MAT_PLAIN, 0x3, st);
    }
    dev_free(tmp);
    return rc;
  }
  Pos p{};
  p.k = op.k;
  for (int j = 0; j < op.k; ++j) p.p[j] = op.pos[j];
  const int d = 1 << op.k;
  for (int pass = 0; pass < (is_dm ? 2 : 1); ++pass) {
    int mode;
    if (pass == 0) {
      mode = dagger ? MAT_ADJOINT : MAT_PLAIN;
    } else {
      mode = dagger ? MAT_TRANSPOSE : MAT_CONJ;
      for (int j = 0; j < op.k; ++j) p.p[j] = op.pos[j] + n;
    }
    int rc;
    if (op.cls == CLS_DIAG) {
      rc = launch_diag(v, elems, nsamples, p, m, ms, mode, op.active, st);
    } else if (op.cls == CLS_MONO) {
      // Adjoint/transpose of a monomial moves entries back along sigma^-1.
      const int* sg = (mode == MAT_ADJOINT || mode == MAT_TRANSPOSE) ? op.sigma_inv : op.sigma;
      rc = launch_monomial(v, elems, nsamples, p, m, ms, mode, sg, d, st);
    } else {
      rc = launch_dense_block(v, elems, nsamples, p, m, ms, mode, g_ctx.tensor_plain, st);
    }
    if (rc) return rc;
  }
  return MB_OK;
}

int apply_plain(mb_circuit c, mb_state s, int64_t mrow_stride) {
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  for (const COp& op : c->ops) {
    int rc = plain_op(c, op, s->d, s->n, is_dm, s->batch, mrow_stride, false);
    if (rc) return rc;
  }
  return MB_OK;
}

int validate_apply(mb_circuit c, mb_state s) {
  if (s->n != c->n) {
    set_error("circuit compiled for %d qubits applied to a %d-qubit state", c->n, s->n);
    return MB_EINVAL;
  }
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  if (c->has_channel && !is_dm) {
    set_error("a channel needs a density-matrix state; convert the state vector first");
    return MB_EUNSUPPORTED;
  }
  return MB_OK;
}

}  // namespace mb

extern "C" int mb_apply(mb_circuit c, mb_state s, const double* theta, size_t ntheta, int flags) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!c || !s || (!theta && ntheta)) return MB_EINVAL;
  if (int rc = validate_apply(c, s)) return rc;
  const bool per_sample = flags & MB_APPLY_PER_SAMPLE;
  if (per_sample && s->kind < MB_BATCH_PURE) {
    set_error("per-sample parameters need a batch state");
    return MB_EINVAL;
  }
  const int rows = per_sample ? s->batch : 1;
  if (rows == 0) return MB_OK;
  if (flags & MB_APPLY_DEVICE_THETA) {
    if (c->theta_rows != rows) {
      set_error("mb_apply: staged parameters have %d rows, the state needs %d", c->theta_rows, rows);
      return MB_EINVAL;
    }
    if (int rc = bind_launch(c, rows)) return rc;
  } else {
    if (int rc = check_not_capturing("mb_apply without MB_APPLY_DEVICE_THETA")) return rc;
    if (int rc = bind_circuit(c, theta, ntheta, rows)) return rc;
  }
  const int64_t stride = per_sample ? c->table_elems : 0;
  if (flags & MB_APPLY_PLAIN) {
    g_ctx.tensor_plain = (flags & MB_APPLY_TENSOR) != 0;
    const int rc = apply_plain(c, s, stride);
    g_ctx.tensor_plain = false;
    return rc;
  }
  return apply_fused(c, s, stride);
}

// =============================================================================================
// Observables
// =============================================================================================
extern "C" int mb_observable_create(const mb_term* terms, size_t nterms, mb_observable* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_observable_create")) return rc;
  if (!out || (!terms && nterms)) return MB_EINVAL;
  std::unique_ptr<mb_observable_s> o(new mb_observable_s());
  // Group terms by sorted site tuple and sum their dense local matrices
  // (QubitsOperator.data + _get_mat, backends/cpu/operators/utils.jl:8-20).
  std::map<std::vector<int>, std::vector<cd>> keys;
  for (size_t t = 0; t < nterms; ++t) {
    const mb_term& tm = terms[t];
    if (tm.nsites < 0 || tm.nsites > 5) {
      set_error("term %zu: %d sites not supported (at most 5)", t, tm.nsites);
      return MB_EUNSUPPORTED;
    }
    if (!std::isfinite(tm.coeff[0]) || !std::isfinite(tm.coeff[1]) || (tm.nsites && !tm.ops) ||
        (tm.nsites && !finite_mat(tm.ops, size_t(tm.nsites) * 8))) {
      set_error("term %zu: coefficients and operators must be finite", t);
      return MB_EINVAL;
    }
    int idx[5];
    for (int j = 0; j < tm.nsites; ++j) {
      idx[j] = j;
      if (tm.sites[j] < 0) {
        set_error("term %zu: operator positions must be positive", t);
        return MB_EINVAL;
      }
      for (int q = 0; q < j; ++q)
        if (tm.sites[q] == tm.sites[j]) {
          set_error("term %zu: operator positions must be distinct", t);
          return MB_EINVAL;
        }
    }
    std::sort(idx, idx + tm.nsites, [&](int a, int b) { return tm.sites[a] < tm.sites[b]; });
    std::vector<int> key(tm.nsites);
    for (int j = 0; j < tm.nsites; ++j) key[j] = tm.sites[idx[j]];
    const int d = 1 << tm.nsites;
    std::vector<cd> M(size_t(d) * d);
    for (int r = 0; r < d; ++r)
      for (int q = 0; q < d; ++q) {
        cd x(tm.coeff[0], tm.coeff[1]);
        for (int j = 0; j < tm.nsites; ++j) {
          const double* op = tm.ops + 8 * idx[j];
          int rb = (r >> j) & 1, qb = (q >> j) & 1;
          x *= cd(op[2 * (rb + 2 * qb)], op[2 * (rb + 2 * qb) + 1]);
        }
        M[r + q * d] = x;
      }
    auto it = keys.find(key);
    if (it == keys.end()) {
      keys[key] = M;
    } else {
      for (size_t e = 0; e < M.size(); ++e) it->second[e] += M[e];
    }
    for (int s : key) o->max_site = std::max(o->max_site, s);
  }
  std::vector<double2> mats;
  bool herm = true;
  for (auto& kv : keys) {
    OKey k{};
    k.k = int(kv.first.size());
    for (int j = 0; j < k.k; ++j) k.pos[j] = kv.first[j];
    k.mat_off = int(mats.size());
    const int d = 1 << k.k;
    for (int r = 0; r < d; ++r)
      for (int q = 0; q < d; ++q)
        if (std::abs(kv.second[r + q * d] - std::conj(kv.second[q + r * d])) > 1e-12 * (1 + std::abs(kv.second[r + q * d])))
          herm = false;
    for (auto& x : kv.second) mats.push_back(d2(x));
    o->keys.push_back(k);
  }
  o->hermitian = herm;
  o->h_mats = mats;
  if (!mats.empty()) {
    int rc = dev_alloc((void**)&o->d_mats, sizeof(double2) * mats.size());
    if (rc) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(o->d_mats, mats.data(), sizeof(double2) * mats.size(), cudaMemcpyHostToDevice,
                                  g_ctx.stream));
    MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  }
  if (int rc = pauli_compile(o.get(), terms, nterms)) return rc;
  *out = o.release();
  return MB_OK;
}

extern "C" int mb_observable_free(mb_observable o) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!o) return MB_OK;
  if (g_ctx.init) {
    dev_free(o->d_mats);
    pauli_free(o);
  }
  delete o;
  return MB_OK;
}

namespace mb {

// <H> per sample into g_ctx.results[0..B-1] (device) using the dense-key kernels.
int expect_keys(mb_observable o, mb_state s, double2* out) {
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  cudaStream_t st = g_ctx.stream;
  if (!out) out = g_ctx.results;
  MB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * s->batch, st));
  for (const OKey& k : o->keys) {
    ReduceOut ro{out, nullptr, nullptr, 1};
    Pos p{};
    p.k = k.k;
    for (int j = 0; j < k.k; ++j) p.p[j] = k.pos[j];
    const double2* m = o->d_mats + k.mat_off;
    int rc;
    if (k.k == 0) {
      rc = is_dm ? launch_dm_trace0(s->d, s->n, s->batch, m, ws(), ro, st)
                 : launch_cross_dense(s->d, s->d, s->elems, s->batch, p, m, 0, MAT_PLAIN, ws(), 0, ro, st);
    } else if (is_dm) {
      rc = launch_dm_trace(s->d, s->n, s->batch, p, m, ws(), 0, ro, st);
    } else {
      rc = launch_cross_dense(s->d, s->d, s->elems, s->batch, p, m, 0, MAT_PLAIN, ws(), 0, ro, st);
    }
    if (rc) return rc;
  }
  return MB_OK;
}

int validate_observable(mb_observable o, mb_state s) {
  if (o->max_site >= s->n && !o->keys.empty() && !(o->keys.size() == 1 && o->keys[0].k == 0)) {
    set_error("observable acts on qubit %d of a %d-qubit state", o->max_site + 1, s->n);
    return MB_EINVAL;
  }
  return MB_OK;
}

}  // namespace mb

extern "C" int mb_expect(mb_observable o, mb_state s, double* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_expect")) return rc;
  if (!o || !s || !out) return MB_EINVAL;
  if (int rc = validate_observable(o, s)) return rc;
  if (s->batch == 0) return MB_OK;
  if (s->batch > 65536) {
    set_error("at most 65536 samples per expectation call");
    return MB_EUNSUPPORTED;
  }
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  const bool keys_only = getenv("MB_EXPECT_KEYS") && atoi(getenv("MB_EXPECT_KEYS")) != 0;
  int rc = (!is_dm && o->pauli_ok && !keys_only) ? expect_pauli(o, s) : expect_keys(o, s);
  if (rc) return rc;
  MB_CHECK_CUDA(cudaMemcpyAsync(out, g_ctx.results, sizeof(double2) * s->batch, cudaMemcpyDeviceToHost, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

namespace mb {
int observable_apply(mb_observable o, const double2* in, double2* out, int n, int is_dm, int nsamples) {
  const int64_t elems = is_dm ? (int64_t(1) << (2 * n)) : (int64_t(1) << n);
  if (o->keys.empty()) {
    MB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * elems * nsamples, g_ctx.stream));
    return MB_OK;
  }
  bool first = true;
  for (const OKey& k : o->keys) {
    Pos p{};
    p.k = k.k;
    for (int j = 0; j < k.k; ++j) p.p[j] = k.pos[j];
    int rc = launch_obs_apply(in, out, elems, nsamples, p, o->d_mats + k.mat_off, first ? 1 : 0, g_ctx.stream);
    if (rc) return rc;
    first = false;
  }
  return MB_OK;
}
}  // namespace mb

extern "C" int mb_observable_apply(mb_observable o, mb_state in, mb_state out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!o || !in || !out) return MB_EINVAL;
  if (in->kind != out->kind || in->n != out->n || in->batch != out->batch || in == out) {
    set_error("observable action needs a distinct output state of the input's shape");
    return MB_EINVAL;
  }
  if (int rc = validate_observable(o, in)) return rc;
  const int is_dm = in->kind == MB_DENSITY || in->kind == MB_BATCH_DENSITY;
  if (!is_dm && o->pauli_ok && !g_ctx.capturing) {
    // pure states from 10 qubits: Pauli-string passes over shared-memory tiles
    bool done = false;
    if (int rc = pauli_apply(o, in->d, out->d, in->n, in->batch, 1.0, &done)) return rc;
    if (done) return MB_OK;
  }
  return observable_apply(o, in->d, out->d, in->n, is_dm, in->batch);
}

// =============================================================================================
// Readout
// =============================================================================================
extern "C" int mb_probabilities(mb_state s, const int* qubits, int nq, double* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_probabilities")) return rc;
  if (!s || !out || nq < 0 || (nq && !qubits)) return MB_EINVAL;
  // _readout_qubits (probabilities.jl:1-6)
  for (int j = 0; j < nq; ++j) {
    if (qubits[j] < 0 || qubits[j] >= s->n) {
      set_error("readout qubit out of range");
      return MB_EINVAL;
    }
    for (int q = 0; q < j; ++q)
      if (qubits[q] == qubits[j]) {
        set_error("readout qubits must be distinct");
        return MB_EINVAL;
      }
  }
  if (s->batch == 0) return MB_OK;
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  const int64_t M = int64_t(1) << nq;
  const size_t bytes = sizeof(double) * M * s->batch;
  double* d_out = nullptr;
  int rc = dev_alloc((void**)&d_out, bytes);
  if (rc) return rc;
  cudaStream_t st = g_ctx.stream;
  const double tol = std::sqrt(2.220446049250313e-16);  // _probability_tolerance (probabilities.jl:16-21)
  MB_CHECK_CUDA(cudaMemsetAsync(d_out, 0, bytes, st));
  MB_CHECK_CUDA(cudaMemsetAsync(g_ctx.flags, 0, sizeof(unsigned) * 2, st));
  rc = launch_marginal(s->d, s->n, is_dm, s->batch, qubits, nq, d_out, g_ctx.flags, tol, st);
  unsigned flags[2] = {0, 0};
  if (!rc) {
    cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(flags, g_ctx.flags, sizeof(flags), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      set_error("probabilities: %s", cudaGetErrorString(e));
      rc = MB_EDEVICE;
    }
  }
  dev_free(d_out);
  if (rc) return rc;
  if (flags[0]) {
    set_error("density-matrix diagonal must be real");
    return MB_ENORM;
  }
  if (flags[1]) {
    set_error("density-matrix probabilities must be nonnegative");
    return MB_ENORM;
  }
  // _normalize_probabilities! (probabilities.jl:23-32)
  for (int b = 0; b < s->batch; ++b) {
    double* p = out + int64_t(b) * M;
    double mn = p[0], total = 0;
    for (int64_t r = 0; r < M; ++r) {
      if (!std::isfinite(p[r])) {
        set_error("probabilities must be finite");
        return MB_ENORM;
      }
      mn = std::min(mn, p[r]);
    }
    if (mn < -tol) {
      set_error("probabilities must be nonnegative");
      return MB_ENORM;
    }
    for (int64_t r = 0; r < M; ++r) {
      p[r] = std::max(p[r], 0.0);
      total += p[r];
    }
    if (!(std::fabs(total - 1) <= std::max(tol, tol * std::max(std::fabs(total), 1.0)))) {
      set_error("state probabilities must sum to one; normalize the state first (sum = %.17g)", total);
      return MB_ENORM;
    }
    for (int64_t r = 0; r < M; ++r) p[r] /= total;
  }
  return MB_OK;
}
