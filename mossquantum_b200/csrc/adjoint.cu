// Adjoint reverse sweep (src/differentiation/circuit.jl:77-229, expectation.jl:4-73,
// objectives.jl:183-296, batch.jl:35-204).
//
// Forward: the circuit runs on a private copy of the initial state; the state at the start
// of every checkpointed segment of k instructions is kept in HBM. Reverse: per instruction
//   gate     Δ <- U'Δ (U'ΔU on density matrices), y <- U'y, and for every active parameter
//            g += Re<y|D|Δ>  (pure)  or  Re(<Δ, D'y> + <Δ, yD>)  (density), D = (dU)'U;
//   channel  Δ <- S'Δ and y <- the channel's input, recomputed from the segment checkpoint
//            (the reference keeps every channel input; recomputation bounds the memory to
//            one checkpoint per segment plus the channel inputs of one segment).
// Circuits with channels run on density matrices throughout (a pure initial state is
// promoted first, DensityMatrix(psi), execution/channels.jl:19); this gives the same
// parameter gradient as promoting at the first channel.
// Fused paths: pure states (one sample) and density matrices (samples with shared parameters)
// run the reverse as dual-state passes (y and Δ tiles together, gradients accumulated in the
// pass). On density matrices a single-qubit channel is reversed by S' on Δ and S^-1 on y (the
// input is uncomputed instead of recomputed); segments keep the product of ||S^-1||_2 within
// 100 and y is reset to the segment's checkpoint after each, which bounds the rounding error.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <vector>

#include "internal.h"

using namespace mb;

namespace {

// Owns one device buffer for the duration of an adjoint call.
struct Buf {
  double2* p = nullptr;
  Buf() = default;
  Buf(const Buf&) = delete;
  ~Buf() { dev_free(p); }
  int alloc(size_t bytes) { return dev_alloc((void**)&p, bytes); }
};

}  // namespace

namespace mb {

// Gradient contribution of one active parameter (generator D at gen_off).
static int gate_gradient(mb_circuit c, const COp& op, const double2* y, const double2* delta, int n, int is_dm,
                         int nsamples, double* d_grad_slot, const double* d_w) {
  Pos p{};
  p.k = op.k;
  for (int j = 0; j < op.k; ++j) p.p[j] = op.pos[j];
  const double2* D = c->d_table + op.gen_off;
  ReduceOut ro{nullptr, d_grad_slot, d_w, 0};
  if (!is_dm) {
    // Re <y| D |Δ> (back_propagate, circuit.jl:136-144)
    return launch_cross_dense(y, delta, int64_t(1) << n, nsamples, p, D, 0, MAT_PLAIN, ws(), 0, ro, g_ctx.stream);
  }
  // Re(<Δ, D' y> + <Δ, y D>) (_density_gate_gradient!, circuit.jl:155-172): D' on the row
  // bits, D^T on the column bits.
  const int64_t elems = int64_t(1) << (2 * n);
  int rc = launch_cross_dense(delta, y, elems, nsamples, p, D, 0, MAT_ADJOINT, ws(), 0, ro, g_ctx.stream);
  if (rc) return rc;
  for (int j = 0; j < op.k; ++j) p.p[j] = op.pos[j] + n;
  return launch_cross_dense(delta, y, elems, nsamples, p, D, 0, MAT_TRANSPOSE, ws(), 0, ro, g_ctx.stream);
}

// Reverse of one application of a unitary circuit c on one pure sample, as used by the serving
// loop for every repetition of an ansatz block. On entry y is the state after c and delta the
// adjoint of the state; on exit y is the state before c, delta = c' delta, and d_grad[slot] has
// been incremented by Re<y|D|delta> per active parameter (back_propagate, circuit.jl:136-144).
// try_fused: use the specialised dual-state passes when the circuit allows them.
int reverse_pure_single(mb_circuit c, int n, double2* y, double2* delta, double* d_grad, bool try_fused,
                        bool* used_fused) {
  if (used_fused) *used_fused = false;
  if (try_fused && n >= 9 && !c->has_channel && !c->ops.empty()) {
    Schedule* S = nullptr;
    if (adjoint_prepare(c, n, 0, int(c->ops.size()), &S) == MB_OK) {
      if (used_fused) *used_fused = true;
      return run_adjoint_schedule(c, S, y, delta, d_grad);
    }
  }
  for (int i = int(c->ops.size()) - 1; i >= 0; --i) {
    const COp& op = c->ops[i];
    int rc;
    if ((rc = plain_op(c, op, delta, n, 0, 1, 0, true))) return rc;
    if ((rc = plain_op(c, op, y, n, 0, 1, 0, true))) return rc;
    if (op.gen_off >= 0 && (rc = gate_gradient(c, op, y, delta, n, 0, 1, d_grad + op.slot, nullptr))) return rc;
  }
  return MB_OK;
}

// Segment length of the two-level recomputation in reverse_dm_single and the number of
// scratch states it needs: one working state, the checkpoints of segments 1.., and the
// channel inputs of the longest segment.
void dm_reverse_plan(mb_circuit c, int* seg_len, int* nscratch) {
  const int k = int(c->ops.size());
  const int m = std::max(1, int(std::ceil(std::sqrt(double(std::max(k, 1))))));
  const int nseg = std::max(1, (k + m - 1) / m);
  int maxch = 0;
  for (int s = 0; s < nseg; ++s) {
    int ch = 0;
    for (int i = s * m; i < std::min(k, (s + 1) * m); ++i) ch += c->ops[i].kind == MB_OP_CHANNEL;
    maxch = std::max(maxch, ch);
  }
  *seg_len = m;
  *nscratch = 1 + (nseg - 1) + maxch;
}

// Forward application of instructions [lo, hi) of c on one density matrix with the plain
// kernels: the segments are about sqrt(k) instructions long, and a fused schedule (with its
// specialised kernels) per distinct segment would cost more to build than it saves.
static int forward_range_dm(mb_circuit c, int n, int lo, int hi, double2* z) {
  for (int i = lo; i < hi; ++i)
    if (int rc = plain_op(c, c->ops[i], z, n, 1, 1, 0, false)) return rc;
  return MB_OK;
}

// Reverse of one application of circuit c (gates and channels) on one density matrix, for the
// serving loop. ckpt is the state before c (kept by the caller); delta enters as the adjoint
// after c and leaves as the adjoint before c; d_grad[slot] += Re(<delta, D'y> + <delta, yD>)
// per active parameter (_density_gate_gradient!, circuit.jl:155-172). Channel inputs come
// from a two-level recomputation: checkpoints every seg_len instructions, then the inputs of
// one segment at a time, so scratch holds dm_reverse_plan's nscratch states.
int reverse_dm_single(mb_circuit c, int n, const double2* ckpt, double2* delta, double* d_grad,
                      double2* const* scratch) {
  const int k = int(c->ops.size());
  // Fused: the state after c, recomputed from the checkpoint with the fused passes, then one
  // dual-state reverse that uncomputes y through the channels' inverses (when their error
  // growth over c stays within 100).
  {
    double growth = 1.0;
    for (const COp& op : c->ops) growth *= reverse_growth(c, op);
    const char* plain_env = getenv("MB_ADJOINT_PLAIN");
    Schedule *adj = nullptr, *fwd = nullptr;
    if (k > 0 && 2 * n >= 8 && growth <= 100.0 && !(plain_env && atoi(plain_env)) &&
        adjoint_prepare(c, n, 0, k, &adj, 1, 1) == MB_OK && get_schedule_ex(c, n, 1, 0, 0, k, 1, &fwd) == MB_OK) {
      const size_t sbytes = sizeof(double2) * (size_t(1) << (2 * n));
      MB_CHECK_CUDA(cudaMemcpyAsync(scratch[0], ckpt, sbytes, cudaMemcpyDeviceToDevice, g_ctx.stream));
      if (int rc = run_schedule(c, fwd, scratch[0], 1, 0)) return rc;
      return run_adjoint_schedule(c, adj, scratch[0], delta, d_grad);
    }
  }
  int m = 1, nscratch = 1;
  dm_reverse_plan(c, &m, &nscratch);
  const int nseg = std::max(1, (k + m - 1) / m);
  const size_t sbytes = sizeof(double2) * (size_t(1) << (2 * n));
  cudaStream_t st = g_ctx.stream;
  double2* z = scratch[0];
  int rc;
  MB_CHECK_CUDA(cudaMemcpyAsync(z, ckpt, sbytes, cudaMemcpyDeviceToDevice, st));
  for (int s = 1; s < nseg; ++s) {
    if ((rc = forward_range_dm(c, n, (s - 1) * m, s * m, z))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(scratch[s], z, sbytes, cudaMemcpyDeviceToDevice, st));
  }
  double2* const* chin = scratch + nseg;
  for (int s = nseg - 1; s >= 0; --s) {
    const int lo = s * m, hi = std::min(k, (s + 1) * m);
    MB_CHECK_CUDA(cudaMemcpyAsync(z, s == 0 ? ckpt : scratch[s], sbytes, cudaMemcpyDeviceToDevice, st));
    int nch = 0;
    for (int i = lo; i < hi; ++i) {
      if (c->ops[i].kind == MB_OP_CHANNEL) MB_CHECK_CUDA(cudaMemcpyAsync(chin[nch++], z, sbytes, cudaMemcpyDeviceToDevice, st));
      if ((rc = plain_op(c, c->ops[i], z, n, 1, 1, 0, false))) return rc;
    }
    for (int i = hi - 1; i >= lo; --i) {
      const COp& op = c->ops[i];
      if ((rc = plain_op(c, op, delta, n, 1, 1, 0, true))) return rc;
      if (op.kind == MB_OP_CHANNEL) {
        MB_CHECK_CUDA(cudaMemcpyAsync(z, chin[--nch], sbytes, cudaMemcpyDeviceToDevice, st));
        continue;
      }
      if ((rc = plain_op(c, op, z, n, 1, 1, 0, true))) return rc;
      if (op.gen_off >= 0 && (rc = gate_gradient(c, op, z, delta, n, 1, 1, d_grad + op.slot, nullptr))) return rc;
    }
  }
  return MB_OK;
}

}  // namespace mb

extern "C" int mb_adjoint(mb_circuit c, mb_observable o, mb_state init, const double* theta, size_t ntheta,
                          const double* weights, int checkpoint_every, double* value, double* grad) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!c || !o || !init || !value || (!grad && c->nslots) || (!theta && ntheta)) return MB_EINVAL;
  if (init->n != c->n) {
    set_error("circuit compiled for %d qubits, initial state has %d", c->n, init->n);
    return MB_EINVAL;
  }
  if (int rc = validate_observable(o, init)) return rc;
  if (!o->hermitian) {
    set_error("adjoint gradients need a Hermitian observable");
    return MB_EUNSUPPORTED;
  }
  const int B = init->batch;
  if (B < 1) {
    set_error("scalar batch objectives require at least one sample");
    return MB_EINVAL;
  }
  const bool init_dm = init->kind == MB_DENSITY || init->kind == MB_BATCH_DENSITY;
  const int is_dm = (init_dm || c->has_channel) ? 1 : 0;
  const int n = c->n;
  const int64_t elems = is_dm ? (int64_t(1) << (2 * n)) : (int64_t(1) << n);
  const size_t sbytes = sizeof(double2) * size_t(elems) * B;
  cudaStream_t st = g_ctx.stream;
  int rc;
  if ((rc = bind_circuit(c, theta, ntheta, 1))) return rc;

  // Sample weights (the reduction of BatchExpectationObjective, api/objectives.jl:229-244).
  std::vector<double> w(B, init->kind >= MB_BATCH_PURE ? 1.0 / B : 1.0);
  if (weights) {
    for (int b = 0; b < B; ++b) {
      if (!std::isfinite(weights[b])) {
        set_error("weights must be finite");
        return MB_EINVAL;
      }
      w[b] = weights[b];
    }
  }
  Buf d_w, d_grad, y, delta;
  if ((rc = d_w.alloc(sizeof(double) * B)) || (rc = d_grad.alloc(sizeof(double) * std::max(1, c->nslots))) ||
      (rc = y.alloc(sbytes)) || (rc = delta.alloc(sbytes)))
    return rc;
  MB_CHECK_CUDA(cudaMemcpyAsync(d_w.p, w.data(), sizeof(double) * B, cudaMemcpyHostToDevice, st));
  double* d_g = reinterpret_cast<double*>(d_grad.p);
  MB_CHECK_CUDA(cudaMemsetAsync(d_g, 0, sizeof(double) * std::max(1, c->nslots), st));
  if (is_dm && !init_dm) {
    if ((rc = launch_to_density(init->d, y.p, n, B, st))) return rc;
  } else {
    MB_CHECK_CUDA(cudaMemcpyAsync(y.p, init->d, sbytes, cudaMemcpyDeviceToDevice, st));
  }

  // Fused path: pure single states with unitary circuits (specialised dual-state passes).
  const int nops_all = int(c->ops.size());
  const char* plain_env = getenv("MB_ADJOINT_PLAIN");
  if (!is_dm && B == 1 && !c->has_channel && n >= 9 && nops_all > 0 && !(plain_env && atoi(plain_env))) {
    const int kf = checkpoint_every > 0 ? checkpoint_every : nops_all;
    const int Sf = (nops_all + kf - 1) / kf;
    std::vector<Schedule*> adj(Sf, nullptr), fwd(Sf, nullptr);
    bool ok = true;
    for (int s2 = 0; s2 < Sf && ok; ++s2) {
      const int lo = s2 * kf, hi = std::min(nops_all, (s2 + 1) * kf);
      ok = adjoint_prepare(c, n, lo, hi, &adj[s2]) == MB_OK && get_schedule_ex(c, n, 0, 0, lo, hi, 1, &fwd[s2]) == MB_OK;
    }
    if (ok) {
      std::vector<std::unique_ptr<Buf>> ck(Sf);
      for (int s2 = 0; s2 < Sf; ++s2) {
        if (checkpoint_every > 0) {
          ck[s2].reset(new Buf());
          if ((rc = ck[s2]->alloc(sbytes))) return rc;
          MB_CHECK_CUDA(cudaMemcpyAsync(ck[s2]->p, y.p, sbytes, cudaMemcpyDeviceToDevice, st));
        }
        if ((rc = run_schedule(c, fwd[s2], y.p, 1, 0))) return rc;
      }
      mb_state_s view;
      view.kind = MB_PURE;
      view.n = n;
      view.batch = 1;
      view.dim = int64_t(1) << n;
      view.elems = elems;
      view.d = y.p;
      if ((rc = o->pauli_ok ? expect_pauli(o, &view) : expect_keys(o, &view))) return rc;
      double2 r0;
      MB_CHECK_CUDA(cudaMemcpyAsync(&r0, g_ctx.results, sizeof(double2), cudaMemcpyDeviceToHost, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
      *value = w[0] * r0.x;
      bool seeded = false;
      if (o->pauli_ok && (rc = pauli_apply(o, y.p, delta.p, n, 1, 2.0, &seeded))) return rc;
      if (!seeded) {
        if ((rc = observable_apply(o, y.p, delta.p, n, 0, 1))) return rc;
        if ((rc = launch_scale(delta.p, elems, 2.0, st))) return rc;
      }
      for (int s2 = Sf - 1; s2 >= 0; --s2) {
        if ((rc = run_adjoint_schedule(c, adj[s2], y.p, delta.p, d_g))) return rc;
        if (ck[s2]) MB_CHECK_CUDA(cudaMemcpyAsync(y.p, ck[s2]->p, sbytes, cudaMemcpyDeviceToDevice, st));
      }
      std::vector<double> gh(std::max(1, c->nslots));
      if (c->nslots) MB_CHECK_CUDA(cudaMemcpyAsync(gh.data(), d_g, sizeof(double) * c->nslots, cudaMemcpyDeviceToHost, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
      for (int q = 0; q < c->nslots; ++q) grad[q] = w[0] * gh[q];
      return MB_OK;
    }
  }

  // Fused path for density matrices (density initial states, or pure ones promoted because the
  // circuit has channels): dual-state passes that reverse single-qubit channels with their
  // inverses. Segments end at checkpoint_every and wherever the product of the channels'
  // ||S^-1||_2 would pass 100, so the rounding error of the uncomputed y stays bounded; y is
  // reset to the segment's checkpoint after each reversed segment. Shared parameters with
  // uniform sample weights (the gradient sums over the samples and is scaled once).
  bool uniform_w = true;
  for (int b = 1; b < B; ++b) uniform_w = uniform_w && w[b] == w[0];
  if (is_dm && uniform_w && 2 * n >= 8 && nops_all > 0 && !(plain_env && atoi(plain_env))) {
    std::vector<int> cuts = {0};
    bool ok = true;
    double growth = 1.0;
    int seg_start = 0;
    for (int i = 0; i < nops_all && ok; ++i) {
      const double gr = reverse_growth(c, c->ops[i]);
      if (!std::isfinite(gr)) {
        ok = false;
        break;
      }
      const bool by_k = checkpoint_every > 0 && i - seg_start >= checkpoint_every;
      if (i > seg_start && (by_k || growth * gr > 100.0)) {
        cuts.push_back(i);
        seg_start = i;
        growth = 1.0;
      }
      growth *= gr;
    }
    cuts.push_back(nops_all);
    const int Sd = int(cuts.size()) - 1;
    std::vector<Schedule*> adj(Sd, nullptr), fwd(Sd, nullptr);
    for (int s2 = 0; s2 < Sd && ok; ++s2)
      ok = adjoint_prepare(c, n, cuts[s2], cuts[s2 + 1], &adj[s2], 1, B) == MB_OK &&
           get_schedule_ex(c, n, 1, 0, cuts[s2], cuts[s2 + 1], B, &fwd[s2]) == MB_OK;
    if (ok) {
      std::vector<std::unique_ptr<Buf>> ck(Sd);
      for (int s2 = 0; s2 < Sd; ++s2) {
        if (s2 > 0 || Sd > 1) {
          ck[s2].reset(new Buf());
          if ((rc = ck[s2]->alloc(sbytes))) return rc;
          MB_CHECK_CUDA(cudaMemcpyAsync(ck[s2]->p, y.p, sbytes, cudaMemcpyDeviceToDevice, st));
        }
        if ((rc = run_schedule(c, fwd[s2], y.p, B, 0))) return rc;
      }
      mb_state_s view;
      view.kind = init->kind >= MB_BATCH_PURE ? MB_BATCH_DENSITY : MB_DENSITY;
      view.n = n;
      view.batch = B;
      view.dim = int64_t(1) << n;
      view.elems = elems;
      view.d = y.p;
      if ((rc = expect_keys(o, &view))) return rc;
      std::vector<double2> r(B);
      MB_CHECK_CUDA(cudaMemcpyAsync(r.data(), g_ctx.results, sizeof(double2) * B, cudaMemcpyDeviceToHost, st));
      // seed: z H' applied to the identity, the dense matrix H per sample (expectation.jl:69-73)
      {
        Buf ident;
        if ((rc = ident.alloc(sbytes))) return rc;
        if ((rc = launch_identity_density(ident.p, n, B, st))) return rc;
        if ((rc = observable_apply(o, ident.p, delta.p, n, 1, B))) return rc;
        MB_CHECK_CUDA(cudaStreamSynchronize(st));
      }
      double v = 0;
      for (int b = 0; b < B; ++b) v += w[b] * r[b].x;
      *value = v;
      for (int s2 = Sd - 1; s2 >= 0; --s2) {
        if ((rc = run_adjoint_schedule(c, adj[s2], y.p, delta.p, d_g))) return rc;
        if (s2 > 0 && ck[s2]) MB_CHECK_CUDA(cudaMemcpyAsync(y.p, ck[s2]->p, sbytes, cudaMemcpyDeviceToDevice, st));
      }
      std::vector<double> gh(std::max(1, c->nslots));
      if (c->nslots) MB_CHECK_CUDA(cudaMemcpyAsync(gh.data(), d_g, sizeof(double) * c->nslots, cudaMemcpyDeviceToHost, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
      for (int q = 0; q < c->nslots; ++q) grad[q] = w[0] * gh[q];
      return MB_OK;
    }
  }

  // Segments of k instructions; checkpoint where a segment holds a channel or k was given.
  const int nops = int(c->ops.size());
  int k = checkpoint_every;
  if (k <= 0) k = c->has_channel ? std::max(1, int(std::ceil(std::sqrt(double(std::max(nops, 1)))))) : std::max(nops, 1);
  const int S = std::max(1, (nops + k - 1) / k);
  std::vector<std::unique_ptr<Buf>> ckpt(S);
  std::vector<char> seg_channel(S, 0);
  for (int i = 0; i < nops; ++i)
    if (c->ops[i].kind == MB_OP_CHANNEL) seg_channel[i / k] = 1;

  // Forward pass.
  for (int s = 0; s < S; ++s) {
    if (checkpoint_every > 0 || seg_channel[s]) {
      ckpt[s].reset(new Buf());
      if ((rc = ckpt[s]->alloc(sbytes))) return rc;
      MB_CHECK_CUDA(cudaMemcpyAsync(ckpt[s]->p, y.p, sbytes, cudaMemcpyDeviceToDevice, st));
    }
    for (int i = s * k; i < std::min(nops, (s + 1) * k); ++i)
      if ((rc = plain_op(c, c->ops[i], y.p, n, is_dm, B, 0, false))) return rc;
  }

  // Observation: value and seed (expectation.jl:4-73).
  {
    mb_state_s view;
    view.kind = is_dm ? (init->kind >= MB_BATCH_PURE ? MB_BATCH_DENSITY : MB_DENSITY)
                      : (init->kind >= MB_BATCH_PURE ? MB_BATCH_PURE : MB_PURE);
    view.n = n;
    view.batch = B;
    view.dim = int64_t(1) << n;
    view.elems = elems;
    view.d = y.p;
    if ((rc = expect_keys(o, &view))) return rc;
    std::vector<double2> r(B);
    MB_CHECK_CUDA(cudaMemcpyAsync(r.data(), g_ctx.results, sizeof(double2) * B, cudaMemcpyDeviceToHost, st));
    MB_CHECK_CUDA(cudaStreamSynchronize(st));
    double v = 0;
    for (int b = 0; b < B; ++b) v += w[b] * r[b].x;
    *value = v;
  }
  if (!is_dm) {
    // λ = (conj z) Hψ + z H'ψ = 2Hψ for Hermitian H and z = 1.
    if ((rc = observable_apply(o, y.p, delta.p, n, 0, B))) return rc;
    if ((rc = launch_scale(delta.p, elems * B, 2.0, st))) return rc;
  } else {
    // z H' applied to the identity: the dense matrix H per sample.
    Buf ident;
    if ((rc = ident.alloc(sbytes))) return rc;
    if ((rc = launch_identity_density(ident.p, n, B, st))) return rc;
    if ((rc = observable_apply(o, ident.p, delta.p, n, 1, B))) return rc;
    MB_CHECK_CUDA(cudaStreamSynchronize(st));
  }

  // Reverse pass.
  for (int s = S - 1; s >= 0; --s) {
    const int lo = s * k, hi = std::min(nops, (s + 1) * k);
    std::vector<std::unique_ptr<Buf>> chin(hi - lo);
    if (seg_channel[s]) {
      Buf z;
      if ((rc = z.alloc(sbytes))) return rc;
      MB_CHECK_CUDA(cudaMemcpyAsync(z.p, ckpt[s]->p, sbytes, cudaMemcpyDeviceToDevice, st));
      for (int i = lo; i < hi; ++i) {
        if (c->ops[i].kind == MB_OP_CHANNEL) {
          chin[i - lo].reset(new Buf());
          if ((rc = chin[i - lo]->alloc(sbytes))) return rc;
          MB_CHECK_CUDA(cudaMemcpyAsync(chin[i - lo]->p, z.p, sbytes, cudaMemcpyDeviceToDevice, st));
        }
        if ((rc = plain_op(c, c->ops[i], z.p, n, is_dm, B, 0, false))) return rc;
      }
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
    }
    for (int i = hi - 1; i >= lo; --i) {
      const COp& op = c->ops[i];
      if (op.kind == MB_OP_CHANNEL) {
        if ((rc = plain_op(c, op, delta.p, n, is_dm, B, 0, true))) return rc;
        MB_CHECK_CUDA(cudaMemcpyAsync(y.p, chin[i - lo]->p, sbytes, cudaMemcpyDeviceToDevice, st));
        continue;
      }
      if ((rc = plain_op(c, op, delta.p, n, is_dm, B, 0, true))) return rc;
      if ((rc = plain_op(c, op, y.p, n, is_dm, B, 0, true))) return rc;
      if (op.gen_off >= 0)
        if ((rc = gate_gradient(c, op, y.p, delta.p, n, is_dm, B, d_g + op.slot, reinterpret_cast<const double*>(d_w.p)))) return rc;
    }
    if (ckpt[s]) MB_CHECK_CUDA(cudaMemcpyAsync(y.p, ckpt[s]->p, sbytes, cudaMemcpyDeviceToDevice, st));
    MB_CHECK_CUDA(cudaStreamSynchronize(st));
    chin.clear();
    ckpt[s].reset();
  }
  if (c->nslots) MB_CHECK_CUDA(cudaMemcpyAsync(grad, d_g, sizeof(double) * c->nslots, cudaMemcpyDeviceToHost, st));
  MB_CHECK_CUDA(cudaStreamSynchronize(st));
  return MB_OK;
}
