// Internal host-side structures of libmossb200 (handles behind the opaque ABI types).
#pragma once
#include <map>
#include <mutex>
#include <vector>

#include "kernels.h"

namespace mb {

enum OpClass { CLS_DENSE = 0, CLS_DIAG = 1, CLS_MONO = 2 };

// One compiled instruction: positions sorted ascending, matrix stored in ordered form in
// the circuit's matrix table (ordered_positions / ordered_mat, abstract_gates.jl:88-112).
struct COp {
  int kind;            // MB_OP_GATE / MB_OP_CHANNEL
  int k;               // number of positions (channel: qubits; its supermatrix spans 2k bits)
  int pos[5];          // ordered positions
  int family, slot, flags;
  double value;
  bool parametric;     // matrix evaluated on the device from theta
  int cls;             // OpClass
  uint32_t active;     // CLS_DIAG: local indices whose factor may differ from 1
  int sigma[32];       // CLS_MONO: destination of local index a (-1 = unchanged)
  int sigma_inv[32];
  int mat_off;         // ordered matrix (gates) or supermatrix (channels) in the table
  int gen_off;         // derivative generator (active parametric gates) or -1
};

struct Schedule;       // fused-pass schedule (fused.cu)

struct mb_circuit_impl_tag {};

}  // namespace mb

struct mb_state_s {
  int kind = 0, n = 0, batch = 1;
  int64_t dim = 1, elems = 1;
  double2* d = nullptr;
  size_t bytes = 0;
};

struct mb_circuit_s {
  uint64_t uid = 0;                   // process-unique id (never reused, unlike the address)
  int n = 0;
  std::vector<mb::COp> ops;
  int nslots = 0;
  bool has_channel = false;
  std::vector<double2> fixed_table;   // one sample's table with fixed matrices filled in
  int64_t table_elems = 1;            // double2 entries per sample row
  std::vector<mb::BindRec> binds;
  mb::BindRec* d_binds = nullptr;
  double2* d_table = nullptr;
  int table_rows = 1;
  double* d_theta = nullptr;
  size_t theta_cap = 0;
  double* h_theta = nullptr;          // pinned staging for theta uploads
  size_t h_theta_cap = 0;
  int theta_rows = 0;                 // rows staged by the last theta upload
  std::vector<mb::Schedule*> scheds;  // fused schedules, built lazily per state shape
};

namespace mb {
struct OKey {
  int k;
  int pos[5];
  int mat_off;
};
struct PauliData;    // pauli.cu
}  // namespace mb

struct mb_observable_s {
  std::vector<mb::OKey> keys;         // one dense local matrix per sorted site tuple
  std::vector<double2> h_mats;
  double2* d_mats = nullptr;
  bool hermitian = true;
  int max_site = -1;
  // Pauli-string form for the fused expectation kernel (pauli.cu).
  bool pauli_ok = false;
  mb::PauliData* pauli = nullptr;
};

namespace mb {

struct Ctx {
  bool init = false;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  size_t budget = 0, used = 0;
  std::map<void*, size_t> sizes;
  double2* partials = nullptr;
  unsigned* counters = nullptr;
  int64_t partials_cap = 0;
  int ncounters = 0;
  double2* results = nullptr;
  unsigned* flags = nullptr;
  bool capturing = false;           // the library stream is recording a CUDA graph
  bool tensor_plain = false;        // per-gate path: dense 4-5 qubit ops on the tensor cores
};

// Dense 4-5 qubit operators through K5 when allowed (MB_DMMA=0 disables it), else K0.
int launch_dense_block(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* m, int64_t mstride,
                       int mode, bool allow_tensor, cudaStream_t st);

extern Ctx g_ctx;
extern std::recursive_mutex g_mu;

int dev_alloc(void** p, size_t bytes);
void dev_free(void* p);
int check_init();
ReduceWs ws();

int state_alloc(int kind, int n, int batch, mb_state* out);
int bind_circuit(mb_circuit c, const double* theta, size_t ntheta, int rows);
int theta_stage(mb_circuit c, const double* theta, size_t ntheta, int rows);
int bind_launch(mb_circuit c, int rows);
int check_not_capturing(const char* what);
int plain_op(mb_circuit c, const COp& op, double2* v, int n, int is_dm, int nsamples, int64_t mrow_stride,
             bool dagger);
int circuit_clone(mb_circuit src, mb_circuit* out);
int circuit_compile_host(const mb_op* ops, size_t nops, int n, mb_circuit c);
void circuit_release(mb_circuit c);
uint64_t next_circuit_uid();
int servers_running();  // serve.cu
int apply_plain(mb_circuit c, mb_state s, int64_t mrow_stride);
int validate_apply(mb_circuit c, mb_state s);
int validate_observable(mb_observable o, mb_state s);
int expect_keys(mb_observable o, mb_state s, double2* out = nullptr);
int observable_apply(mb_observable o, const double2* in, double2* out, int n, int is_dm, int nsamples);

// fused.cu
int apply_fused(mb_circuit c, mb_state s, int64_t mrow_stride);
bool jit_sizes(int nbits);  // register sizes that run on the specialised (NVRTC) kernels
int get_schedule_ex(mb_circuit c, int n, int dm, int adjoint, int lo, int hi, int nsamples, Schedule** out);
int run_schedule(mb_circuit c, Schedule* S, double2* v, int nsamples, int64_t mstride);
int run_adjoint_schedule(mb_circuit c, Schedule* S, double2* y, double2* d, double* d_grad);
// dm: the range runs on density matrices (single-qubit channels reversed with their inverses);
// nsamples: samples stored back to back that share the parameters.
int adjoint_prepare(mb_circuit c, int n, int lo, int hi, Schedule** out, int dm = 0, int nsamples = 1);
// Growth factor of rounding errors in y when a reverse sweep uncomputes through op (1 for
// gates, ||S^-1||_2 for a single-qubit channel, infinity if it cannot be inverted).
double reverse_growth(mb_circuit c, const COp& op);
void release_schedules(mb_circuit c);

// adjoint.cu: single-sample reverse sweeps of one circuit application (serving loop)
int reverse_pure_single(mb_circuit c, int n, double2* y, double2* delta, double* d_grad, bool try_fused,
                        bool* used_fused);
void dm_reverse_plan(mb_circuit c, int* seg_len, int* nscratch);
int reverse_dm_single(mb_circuit c, int n, const double2* ckpt, double2* delta, double* d_grad,
                      double2* const* scratch);

// pauli.cu
int pauli_compile(mb_observable o, const mb_term* terms, size_t nterms);
void pauli_free(mb_observable o);
int expect_pauli(mb_observable o, mb_state s, double2* out = nullptr);
// Whether Pauli programs built on the calling thread may compile specialised kernels (default
// yes); when not, they run on the interpreter kernel.
void pauli_allow_compile(bool on);
int pauli_apply(mb_observable o, const double2* in, double2* out, int n, int nsamples, double scale, bool* done);

}  // namespace mb
