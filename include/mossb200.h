/*
 * mossb200.h - C ABI of the B200 dense simulation backend for MOSSQuantum.
 *
 * The library owns device-resident quantum states (ComplexF64, interleaved re/im, the
 * same byte layout as Julia's Vector{ComplexF64}) and runs every numerical step on one
 * NVIDIA B200 (sm_100a). The host-side backend (a Julia package through `ccall`, or the
 * Python package mossquantum_b200 through ctypes) calls only these functions.
 *
 * Conventions (identical to MOSSQuantum, docs/conventions.md:5-17):
 *   - qubit positions are ZERO-based here (reference position q is bit q-1);
 *     bit 0 is the least significant bit of the amplitude index;
 *   - a gate matrix's first position is its least significant local bit;
 *   - matrices are column-major, complex interleaved (Julia Matrix{ComplexF64});
 *   - density matrices are 2^n x 2^n column-major: row bits are the low n bits of the
 *     vectorised index, column bits the high n bits;
 *   - batch states store B samples back to back, one per column.
 *
 * Every function returns MB_OK (0) or a negative MB_E* code; mb_last_error() returns a
 * thread-local message for the last failure on the calling thread. Validation happens
 * before any device memory is touched, matching the reference's "validate before
 * mutating" rule (src/api/backend_protocols.jl:203-215). There is no CPU fallback:
 * every numerical call runs on the GPU or fails.
 */
#ifndef MOSSB200_H
#define MOSSB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MB_API __attribute__((visibility("default")))
#else
#define MB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define MB_OK 0
#define MB_EINVAL (-1)          /* invalid argument: ArgumentError / DimensionMismatch   */
#define MB_EUNSUPPORTED (-2)    /* UnsupportedOperation / UnsupportedGradient            */
#define MB_ENOMEM_BUDGET (-3)   /* the HBM byte budget would be exceeded                 */
#define MB_ETIMEOUT (-4)        /* a bounded wait ran out (serving loop, persistent work) */
#define MB_EDEVICE (-5)         /* CUDA runtime error                                    */
#define MB_ENOTINIT (-6)        /* mb_init has not been called                           */
#define MB_ENORM (-7)           /* probabilities: state not normalised / negative entry  */
#define MB_ENOTREADY (-8)       /* serving: result not available yet                     */

/* ---- state kinds --------------------------------------------------------------------- */
#define MB_PURE 0            /* StateVector           (src/states/state_vector.jl:12)        */
#define MB_DENSITY 1         /* DensityMatrix         (src/states/density_matrix.jl:12)      */
#define MB_BATCH_PURE 2      /* BatchStateVector      (src/states/batch_state_vector.jl:18)  */
#define MB_BATCH_DENSITY 3   /* BatchDensityMatrix    (src/states/batch_density_matrix.jl:17)*/

/* ---- instruction kinds and gate families ---------------------------------------------- */
#define MB_OP_GATE 0         /* unitary gate (Gate{N}, src/quantum_circuits/gates/)          */
#define MB_OP_CHANNEL 1      /* Kraus channel (QuantumMap, channels/quantum_map.jl:9-36)     */

#define MB_FAM_MATRIX 0      /* fixed matrix given in mb_op.data                             */
#define MB_FAM_RX 1          /* RxGate   Rx(θ)          (gates/Gates.jl:37)                  */
#define MB_FAM_RY 2          /* RyGate   Ry(θ)          (gates/Gates.jl:39)                  */
#define MB_FAM_RZ 3          /* RzGate   Rz(θ)          (gates/Gates.jl:41)                  */
#define MB_FAM_PHASE 4       /* PHASEGate diag(1,e^{iθ}) (gates/Gates.jl:11)                 */
#define MB_FAM_CRX 5         /* CRxGate  CONTROL(Rx(θ)), pos = (control, target)             */
#define MB_FAM_CRY 6         /* CRyGate                                                      */
#define MB_FAM_CRZ 7         /* CRzGate                                                      */
#define MB_FAM_CPHASE 8      /* CPHASEGate CONTROL(PHASE(θ))                                 */
#define MB_FAM_CCPHASE 9     /* CCPHASEGate CONTROLCONTROL(PHASE(θ)), pos = (c1, c2, target) */
#define MB_FAM_SELECT 10     /* one of nkraus operators in data (1-3 positions), chosen by the */
                             /* integer value of its parameter: the branch of a Kraus trajectory */
                             /* (execution/noisy_execution.jl:40-120); not differentiable        */

#define MB_OPF_ADJOINT 1     /* AdjointQuantumGate wrapper (gates/quantum_gate.jl:32-45)     */

/* One instruction of a circuit template (QCircuit element, circuits/circuit.jl:98).
 * pos: zero-based positions in the gate's own order (positions(g)); the library sorts
 * them and permutes the matrix exactly like ordered_positions/ordered_mat
 * (gates/abstract_gates.jl:88-112,162-166).
 * Parametric families take their angle from theta[slot] at apply time (slot >= 0, an
 * active parameter) or from `value` (slot < 0, a frozen parameter). */
typedef struct mb_op {
  int32_t kind;        /* MB_OP_GATE or MB_OP_CHANNEL                                     */
  int32_t nq;          /* number of positions: gates 0..5, channels 1..2                  */
  int32_t pos[5];      /* zero-based qubit positions in the instruction's own order       */
  int32_t family;      /* MB_FAM_*; channels use MB_FAM_MATRIX                            */
  int32_t slot;        /* active-parameter slot (0-based) or -1                           */
  int32_t flags;       /* MB_OPF_*                                                        */
  int32_t nkraus;      /* channels: number of Kraus matrices in data                      */
  int32_t reserved;
  double value;        /* frozen parameter value for parametric families                  */
  const double* data;  /* MATRIX gates: 2^nq x 2^nq; channels: nkraus such matrices       */
} mb_op;

/* One observable term (QubitsTerm, operators/qubits_term.jl:12-30): coeff * ⊗ ops[j] on
 * sites[j]. Sites are zero-based, distinct, in any order; ops are 2x2 column-major. */
typedef struct mb_term {
  int32_t nsites;      /* 0..5 (0 = coeff * identity)                                      */
  int32_t sites[5];
  double coeff[2];     /* complex coefficient (re, im)                                     */
  const double* ops;   /* nsites 2x2 complex matrices, 8 doubles each                      */
} mb_term;

typedef struct mb_state_s* mb_state;
typedef struct mb_circuit_s* mb_circuit;
typedef struct mb_observable_s* mb_observable;

/* apply flags */
#define MB_APPLY_FUSED 0       /* tiled / fused kernels (default)                          */
#define MB_APPLY_PLAIN 1       /* one plain kernel launch per gate (the per-call drop-in)  */
#define MB_APPLY_PER_SAMPLE 2  /* batch states: theta holds B rows of nslots values         */
#define MB_APPLY_TENSOR 8      /* with MB_APPLY_PLAIN: dense 4-5 qubit gates and 2-qubit     */
                               /* channels on the FP64 tensor cores (K5) instead of K0       */

/* ---- context: replaces the CPUBackend singleton (src/api/backend_protocols.jl:10-70) --- */
MB_API int mb_init(int device, size_t hbm_budget_bytes);      /* budget 0 = 90% of free HBM    */
MB_API int mb_shutdown(void);
MB_API const char* mb_last_error(void);
MB_API int mb_memory_info(size_t* used_bytes, size_t* budget_bytes);
MB_API int mb_synchronize(void);
MB_API int mb_version(void);
/* Kernel launches the library has issued since mb_init (for launch accounting). */
MB_API int mb_launch_count(uint64_t* launches);

/* The CUDA stream (cudaStream_t) every library kernel runs on, for event timing and
 * interop; callers must not destroy it. */
MB_API int mb_get_stream(void** stream);

/* Per-kernel timing: when enabled, every launch is bracketed by CUDA events on the library
 * stream and its algorithmic HBM bytes are recorded. mb_profile_report synchronises and
 * fills up to `cap` entries (one per kernel name); *count receives the number of names. */
typedef struct mb_kernel_stat {
  char name[48];
  uint64_t launches;
  double total_ms;
  double bytes;        /* algorithmic bytes summed over launches */
  double flops;        /* algorithmic FP64 flops summed over launches (8*2^k per amplitude */
                       /* for a dense k-qubit complex gate; sign flips and swaps count 0)  */
} mb_kernel_stat;
MB_API int mb_profile(int enable);
MB_API int mb_profile_report(mb_kernel_stat* stats, int cap, int* count);
/* Times a DFMA-only kernel on every SM and returns the FP64 rate it reaches (TFLOP/s):
 * the measured denominator for passes bound by the FP64 pipe. */
MB_API int mb_measure_fp64_peak(double* tflops);

/* ---- states: StateVector / DensityMatrix / batches (src/states/*.jl) ------------------ */
/* Allocate a state of `kind` with n qubits (0..30 pure, 0..15 density) and `batch`
 * samples (ignored for single kinds). Contents are |0...0> (state_vector.jl:36-40). */
MB_API int mb_state_create(int kind, int n, int batch, mb_state* out);
MB_API int mb_state_free(mb_state s);
MB_API int mb_state_set_zero(mb_state s);
MB_API int mb_state_upload(mb_state s, const double* host, size_t n_doubles);
MB_API int mb_state_download(mb_state s, double* host, size_t n_doubles);
MB_API int mb_state_copy(mb_state dst, mb_state src);               /* same kind, n and batch  */
MB_API int mb_state_info(mb_state s, int* kind, int* n, int* batch);
/* DensityMatrix(psi) = psi psi' per sample (execution/channels.jl:19). dst must be the
 * density kind of src's shape. */
MB_API int mb_state_to_density(mb_state src, mb_state dst);
/* Device address of the sample storage (for zero-copy interop; never a host pointer). */
MB_API int mb_state_device_ptr(mb_state s, void** dev_ptr);

/* ---- circuits (QCircuit + bind_parameters, src/api/parameter_binding.jl:19-63) -------- */
MB_API int mb_circuit_create(const mb_op* ops, size_t nops, int n, mb_circuit* out);
MB_API int mb_circuit_free(mb_circuit c);
MB_API int mb_circuit_nslots(mb_circuit c, int* nslots);
/* Number of fused passes the fused schedule uses on an n-qubit pure state. */
MB_API int mb_circuit_passes(mb_circuit c, int* npasses);
/* Host-only schedule of an instruction list (needs no device and no mb_init): the number of
 * passes (tile, register and plain) the fused scheduler makes for an n-qubit pure state
 * (dm = 0) or density matrix (dm = 1) with the given tile and register bits, and whether every
 * fused operation landed in exactly one pass. For tests and capacity planning. */
MB_API int mb_schedule_info(const mb_op* ops, size_t nops, int n, int dm, int tile_bits, int reg_bits, int nsamples,
                            int* npasses, int* ntile, int* nreg, int* nplain, int* complete);
/* Host-only check of the forward lowering (needs no device and no mb_init; a test hook, no
 * counterpart in the reference): lowers a circuit of fixed gates and channels for an n-qubit
 * pure state or density matrix (at most 22 amplitude bits) as the fused schedules do, applies
 * both the compiled instructions and the lowered micro-ops (before scheduling, in the order
 * the scheduled passes run them, and as the passes' encoded register-stage micro-ops) to one
 * seeded random vector on the host, and reports the three maximum deviations. Returns no
 * amplitudes. */
MB_API int mb_lowering_check(const mb_op* ops, size_t nops, int n, int dm, int tile_bits, int reg_bits, uint64_t seed,
                             double* err_ops, double* err_sched, double* err_mops);
/* apply!(circuit, state) (execution/gates.jl:21-36, batch_gates.jl, channels.jl).
 * theta: host array of nslots values (or B*nslots with MB_APPLY_PER_SAMPLE).
 * A circuit with channels requires a density kind (pure states must be promoted first,
 * mirroring StateVector -> DensityMatrix in execution/channels.jl:19). */
MB_API int mb_apply(mb_circuit c, mb_state s, const double* theta, size_t ntheta, int flags);

/* ---- prepared execution: device-side inputs/outputs and CUDA-graph replay ---------------
 * (the B200 counterpart of prepared plans / sweeps, src/execution/execution_plans.jl:12-240).
 * A caller warms a sequence of calls up once (schedules, specialised kernels, buffers), then
 * records it between mb_graph_begin and mb_graph_end and replays it with mb_graph_launch.
 * Inside a recording only calls that neither synchronise nor allocate are allowed: mb_apply
 * with MB_APPLY_DEVICE_THETA, mb_state_set_zero, mb_expect_to_device. */
#define MB_APPLY_DEVICE_THETA 4  /* use the parameters last given to mb_theta_upload        */
MB_API int mb_theta_upload(mb_circuit c, const double* theta, size_t ntheta, int rows);
MB_API int mb_buffer_alloc(size_t bytes, void** dev);
MB_API int mb_buffer_free(void* dev);
MB_API int mb_buffer_download(const void* dev, void* host, size_t bytes);
/* <H> per sample written as complex doubles to device memory (no host synchronisation). */
MB_API int mb_expect_to_device(mb_observable o, mb_state s, double* dev_out);
typedef struct mb_graph_s* mb_graph;
MB_API int mb_graph_begin(void);
MB_API int mb_graph_end(mb_graph* out);
MB_API int mb_graph_launch(mb_graph g);
MB_API int mb_graph_free(mb_graph g);

/* ---- uneven batches in one persistent launch ---------------------------------------------
 * (batches of the reference hold one register size, src/states/batch_state_vector.jl; this is
 * the B200 form of many sizes with per-sample parameters). A plan over groups (circuit g on
 * state g: a pure batch of one register size, its parameters staged with mb_theta_upload, one
 * row per sample) runs every pure group of 8..17 qubits in ONE persistent kernel: CTAs take
 * work items (pass, sample, chunk of tiles) from a work counter, pass by pass, each waiting
 * for its sample's previous pass; the passes run as straight-line code compiled for the plan
 * (NVRTC, at mb_uneven_create), or through the micro-op interpreter without NVRTC (two small
 * launches before it bind the parameter rows and form the fused single-qubit products of every
 * group). Other groups (more qubits, density matrices, instructions a tile cannot hold) run
 * through mb_apply's fused path after it. Circuits and states must outlive the plan.
 * mb_uneven_apply may be recorded into a graph once it has run eagerly. */
typedef struct mb_uneven_s* mb_uneven;
#define MB_UNEVEN_ZERO 1  /* start every sample from |0...0> */
MB_API int mb_uneven_create(const mb_circuit* circuits, const mb_state* states, int ngroups, mb_uneven* out);
MB_API int mb_uneven_apply(mb_uneven u, int flags);
MB_API int mb_uneven_info(mb_uneven u, int* persistent_groups, int* fallback_groups, int* samples);
MB_API int mb_uneven_free(mb_uneven u);

/* ---- tuning: tile bits t (10..12) and register bits R (3..5) per register size ---------- */
MB_API int mb_tuning_set(int nbits, int tile_bits, int reg_bits);
MB_API int mb_tuning_get(int nbits, int* tile_bits, int* reg_bits);
/* Fusion width per register size: 1 (default) multiplies every run of operations on one qubit
 * into one matrix at bind time (2x2 on pure states; on density matrices both gate halves with
 * the channels after them as one 4x4), 0 applies every gate as its own micro-op. */
MB_API int mb_tuning_set_fusion(int nbits, int fusion);
/* Specialised (NVRTC-compiled) pass kernels per register size: 1 always, 0 never, -1 the default
 * (sizes from 18 bits; MB_JIT_MIN_BITS moves the threshold). Prepared plans that replay many
 * times use 1 for smaller sizes, where the compile cost is paid once. */
MB_API int mb_tuning_set_specialised(int nbits, int mode);
MB_API int mb_tuning_get_fusion(int nbits, int* fusion);
/* Times the fused execution of c on s for each candidate (t, R, fusion width) and records the
 * fastest for s's register size; best_ms receives its time per apply. Sizes that run on
 * specialised kernels try 2^10- and 2^11-amplitude tiles with 8 amplitudes per thread and
 * fusion, then the faster of the two without fusion: three sets of kernel compilations. */
MB_API int mb_autotune(mb_circuit c, mb_state s, const double* theta, size_t ntheta, int flags, int* best_t,
                       int* best_r, double* best_ms);

/* ---- observables (QubitsOperator, src/observables/expectation.jl:1-73) ---------------- */
MB_API int mb_observable_create(const mb_term* terms, size_t nterms, mb_observable* out);
MB_API int mb_observable_free(mb_observable o);
/* <H> per sample: out holds 2 doubles (re, im) per sample (1 sample for single kinds). */
MB_API int mb_expect(mb_observable o, mb_state s, double* out);
/* out = H * in (execution/operators.jl:3-63); out has in's kind and shape. */
MB_API int mb_observable_apply(mb_observable o, mb_state in, mb_state out);

/* ---- readout (src/execution/probabilities.jl:42-105) ---------------------------------- */
/* Marginal probabilities on `qubits` (zero-based; the first is the least significant bit
 * of the output index), normalised; out holds 2^nq doubles per sample. */
MB_API int mb_probabilities(mb_state s, const int* qubits, int nq, double* out);

/* ---- measurement and post-selection (src/execution/measurement.jl:4-201,
 *      src/execution/post_selection.jl:3-112) -------------------------------------------
 * w receives 2 doubles per sample: the unnormalised weights of outcome 0 and 1 of `qubit`
 * (sum of |psi_i|^2, or Re rho_ii, over the indices whose bit is 0 / 1); the host normalises
 * them and draws outcomes with its own random stream (discrete_sample, sampling.jl:3-18). */
MB_API int mb_qubit_weights(mb_state s, int qubit, double* w);
/* Collapses sample b onto outcomes[b] and divides by sqrt(probs[b]) (_collapse_batch_column!,
 * measurement.jl); with auto_reset the kept amplitudes move to the qubit's 0 branch. Density
 * matrices get the operator on the row and column bits. Every sample is validated first. */
MB_API int mb_collapse(mb_state s, int qubit, const int* outcomes, const double* probs, int auto_reset);
/* dst (pure, n-1 qubits, same batch) = scales[b] * the outcomes[b] slice of src
 * (_qubit_slice, measurement.jl; post_select without keep, post_selection.jl). */
MB_API int mb_remove_qubit(mb_state src, int qubit, const int* outcomes, const double* scales, mb_state dst);
/* Multiplies sample b by scales[b] (renormalising trajectories, normalize!). */
MB_API int mb_scale_samples(mb_state s, const double* scales);

/* ---- partial trace, inner products, fidelities ------------------------------------------
 * partial_tr (observables/partial_trace.jl:11-97): out = Tr_sites(in) per sample; sites are
 * k distinct zero-based qubits, 0 < k < n; the remaining qubits keep their order as the low
 * bits of out, a DensityMatrix (BatchDensityMatrix for batch inputs) of n - k qubits. A pure
 * input gives V V' (partial_tr(::StateVector), partial_trace.jl:58-71). */
MB_API int mb_partial_trace(mb_state in, const int* sites, int k, mb_state out);
/* <x|y> per sample (dot(x, y), conjugating x) for pure states of equal shape; 2 doubles each. */
MB_API int mb_inner(mb_state x, mb_state y, double* out);
/* <y|rho|y> per sample: fidelity(::DensityMatrix, ::StateVector) (density_matrix.jl:129). */
MB_API int mb_sandwich(mb_state rho, mb_state y, double* out);
/* Copies sample `index` of a batch state into a single state of the same kind and size. */
MB_API int mb_state_extract(mb_state src, int index, mb_state dst);
/* Copies a single state into every sample of a batch state of the same kind and size. */
MB_API int mb_state_broadcast(mb_state src, mb_state dst);
/* dst (batch of copies * B samples) = `copies` back-to-back copies of the batch src. */
MB_API int mb_state_tile(mb_state src, int copies, mb_state dst);

/* ---- adjoint gradients (src/differentiation/objectives.jl:183-296) --------------------
 * value = sum_b w_b Re<H>_b after applying the circuit to a copy of `init`; grad[slot] =
 * d value / d theta[slot] (slots, not independent parameters: the host accumulates a
 * ParameterMap). weights: one per sample (NULL = 1 for single kinds, 1/B for batches).
 * checkpoint_every: forward checkpoints every k instructions (<= 0 picks automatically). */
MB_API int mb_adjoint(mb_circuit c, mb_observable o, mb_state init, const double* theta, size_t ntheta,
               const double* weights, int checkpoint_every, double* value, double* grad);

/* ---- serving: continuous batching of circuit evaluations ------------------------------
 * Replaces the one-call-at-a-time objective evaluation of the reference
 * (evaluate / value_and_gradient, src/api/objectives.jl:15-244,
 * src/differentiation/objectives.jl:183-296) for a stream of independent requests.
 * A request is an ansatz: `repeats` repetitions of a parametrised block circuit (one layer),
 * each repetition with its own parameters, applied to |0...0> of a pure state or a density
 * matrix, followed by <H> and optionally its adjoint gradient.
 * A scheduler thread owned by the library admits requests in arrival order against the
 * server's HBM byte budget (16*2^n per pure state, 16*4^n per density matrix, plus gradient
 * buffers and checkpoints), keeps their states resident, and on every iteration advances
 * every admitted request by one layer: requests of the same block and kind share one
 * batched launch per fused pass with per-sample parameters, gradient requests run one
 * reverse layer each. Requests join and leave between iterations.
 * The block and observable handles of a request must stay valid until it completes. */
typedef struct mb_server_config {
  size_t hbm_budget_bytes;  /* admission budget in bytes; 0 = what the library budget leaves   */
  int max_active;           /* most admitted requests at once; 0 = 4096                         */
  int reserved[7];
} mb_server_config;

typedef struct mb_request {
  mb_circuit block;         /* one layer, compiled for n qubits; its slots are the layer's      */
                            /* parameters (channels require MB_DENSITY)                        */
  mb_observable observable; /* Hermitian for gradient requests                                 */
  int kind;                 /* MB_PURE or MB_DENSITY                                           */
  int repeats;              /* layers, >= 1                                                    */
  const double* theta;      /* repeats * nslots(block) values, layer by layer; copied           */
  size_t ntheta;
  int gradient;             /* 0: <H>; 1: <H> and d Re<H> / d theta (adjoint method)           */
  int reserved[5];
} mb_request;

typedef struct mb_result {
  int status;               /* MB_OK or the request's error code                                */
  int iterations;           /* scheduler iterations the request took part in                   */
  double value[2];          /* <H> (re, im)                                                    */
  double latency_ms;        /* submission to completion                                        */
  double queue_ms;          /* submission to admission                                         */
  char error[128];          /* message when status != MB_OK                                    */
} mb_result;

typedef struct mb_server_stats {
  uint64_t submitted, completed, failed, iterations;
  int active, pending;
  size_t bytes_in_use, peak_bytes, budget_bytes;
  double p50_ms, p99_ms;    /* latency percentiles of the completed requests                   */
  double evals_per_s;       /* completed requests / (last completion - first submission)       */
  double jit_compile_ms;    /* specialised-kernel compile time spent since start / stats reset  */
  uint64_t jit_compiles;    /* kernels compiled since start / stats reset                       */
} mb_server_stats;

typedef struct mb_server_s* mb_server;
MB_API int mb_server_start(const mb_server_config* cfg, mb_server* out);
/* Queues a request; returns at once with its ticket. */
MB_API int mb_submit(mb_server s, const mb_request* req, uint64_t* ticket);
/* MB_ENOTREADY while the request is queued or running; otherwise fills res (and, for
 * gradient requests, grad with repeats*nslots doubles when ngrad is large enough), releases
 * the ticket and returns MB_OK. */
MB_API int mb_poll(mb_server s, uint64_t ticket, mb_result* res, double* grad, size_t ngrad);
/* As mb_poll, waiting up to timeout_ms (< 0: no limit); MB_ETIMEOUT when it runs out. */
MB_API int mb_wait(mb_server s, uint64_t ticket, int timeout_ms, mb_result* res, double* grad, size_t ngrad);
MB_API int mb_server_stats_get(mb_server s, mb_server_stats* out);
/* Clears the latency record and counters (between load levels of a sweep). */
MB_API int mb_server_stats_reset(mb_server s);
/* Finishes the admitted requests, fails the queued ones, joins the scheduler thread and
 * releases the server's memory. Call before mb_shutdown. */
MB_API int mb_server_stop(mb_server s);

/* ---- allocation-free expectation -----------------------------------------------------
 * No counterpart in the reference: MOSSQuantum's CPU path never allocates device memory.
 * For callers that cannot allocate device memory (a pre-planned HBM pool with every byte
 * assigned, a latency-critical path where cudaMalloc/cudaFree would synchronise the GPU,
 * a plug-in that may only use memory its host hands it). It needs no mb_init.
 * <psi_b|M|psi_b> for b = 0..nsamples-1, where M is a 2^k x 2^k column-major complex matrix
 * on `positions` (zero-based, first = least significant local bit) and the samples are
 * nsamples states of 2^n amplitudes stored back to back at device address state_dev.
 * out: 2*nsamples host doubles (re, im). stream: a cudaStream_t (NULL = default stream); the
 * call returns after the result has reached `out`.
 * Limits: k <= 3, nsamples <= 32 (the reduction scratch is a fixed 82,560-byte array in the
 * library, held on every GPU that loads it until exit). The first call on each device looks
 * up that array's device address, so make it before any stream capture; the address is kept
 * for the life of the process, so do not call this after resetting the device
 * (cudaDeviceReset). All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
MB_API int mb_expect_local_noalloc(const double* state_dev, int n, int nsamples, int k, const int* positions,
                                   const double* matrix, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MOSSB200_H */
