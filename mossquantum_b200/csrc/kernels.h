// Launchers for the device kernels of libmossb200 (internal).
#pragma once
#include "common.cuh"

namespace mb {

// Reduction workspace: per-block partial sums plus a "blocks done" counter per slot.
// The last block of a reduction sums the partials in index order (deterministic) and
// resets its counter, so the workspace needs no clearing between launches.
struct ReduceWs {
  double2* partials;     // capacity entries
  unsigned* counters;    // ncounters entries, zero between launches
  int64_t capacity;
  int ncounters;
};

// Where a finished reduction goes.
struct ReduceOut {
  double2* out;          // per-sample complex result (may be null)
  double* grad;          // if non-null: grad[0] += sum_b w[b] * Re(result_b)
  const double* weights; // device weights per sample (null = 1)
  int accumulate;        // out[b] += result instead of out[b] = result
};

// ---- plain per-gate sweeps (K0) and their diagonal / monomial specialisations ----------
// Every gate kernel works on `nsamples` samples of `elems` amplitudes each (the samples
// of a batch state). The matrix of sample b is mats + b * mstride (mstride 0 = shared).
int launch_dense(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* mats,
                 int64_t mstride, int mode, cudaStream_t st);
// Diagonal gate: only the local indices in active_mask are read and rescaled.
int launch_diag(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* mats,
                int64_t mstride, int mode, uint32_t active_mask, cudaStream_t st);
// Monomial gate (permutation times phases): local index a moves to sigma[a] with factor
// m[sigma[a], a]; only the nactive listed local indices move.
int launch_monomial(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* mats,
                    int64_t mstride, int mode, const int* sigma_host, int d, cudaStream_t st);

// Dense 4- or 5-qubit operator on the FP64 tensor cores (K5, dmma.cu); positions ascending,
// one matrix shared by all samples. MB_EUNSUPPORTED when the shape does not fit.
int launch_dmma(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* m, int mode,
                cudaStream_t st);

// ---- state utilities ---------------------------------------------------------------------
int launch_set_basis(double2* v, int64_t elems, int nsamples, int64_t index, cudaStream_t st);
int launch_to_density(const double2* psi, double2* rho, int n, int nsamples, cudaStream_t st);
int launch_identity_density(double2* rho, int n, int nsamples, cudaStream_t st);
int launch_scale(double2* v, int64_t count, double s, cudaStream_t st);

// ---- reductions ------------------------------------------------------------------------------
// sum over blocks of conj(c) (M v) on `pos` (cross expectation <c|M|v>); c may equal v.
int launch_cross_dense(const double2* c, const double2* v, int64_t elems, int nsamples, const Pos& pos,
                       const double2* m, int64_t mstride, int mode, const ReduceWs& ws, int slot,
                       const ReduceOut& ro, cudaStream_t st);
// tr(M rho) for a local M on the row positions of an n-qubit density matrix.
int launch_dm_trace(const double2* rho, int n, int nsamples, const Pos& pos, const double2* m,
                    const ReduceWs& ws, int slot, const ReduceOut& ro, cudaStream_t st);
// s * tr(rho) with s = m[0].
int launch_dm_trace0(const double2* rho, int n, int nsamples, const double2* m, const ReduceWs& ws,
                     const ReduceOut& ro, cudaStream_t st);
// out (+)= M_key * in on pos (observable action); first = overwrite instead of add.
int launch_obs_apply(const double2* in, double2* out, int64_t elems, int nsamples, const Pos& pos,
                     const double2* m, int first, cudaStream_t st);

// ---- readout -------------------------------------------------------------------------------
// Marginal probabilities: out[b * 2^nq + r] = sum of p_i over i whose readout bits form r.
// For density matrices p_i = Re rho_ii; |Im rho_ii| > tol raises flags[0].
int launch_marginal(const double2* v, int n, int is_dm, int nsamples, const int* qubits, int nq,
                    double* out, unsigned* flags, double tol, cudaStream_t st);

// ---- parameter binding -------------------------------------------------------------------------
// One bind record per parametric instruction; the kernel writes its ordered matrix (and the
// derivative generator when gen_off >= 0) for every sample's parameter vector.
struct BindRec {
  int family;
  int flags;
  int slot;
  int k;
  double value;
  int mat_off;        // offset of the ordered matrix in one sample's matrix table (double2)
  int gen_off;        // offset of the ordered generator, or -1
  int perm[8];        // ordered local index a' -> own-order local index (k <= 3)
  int nopt;           // MB_FAM_SELECT: number of stored operators (ordered, after the matrix)
};
int launch_bind(const BindRec* recs_dev, int nrecs, const double* theta_dev, int nslots, int ntheta_rows,
                double2* table, int64_t table_stride, cudaStream_t st);

}  // namespace mb
