/*
 * vqc_b200.h -- C ABI of libvqcb200.so, the B200 (sm_100a) engine for the
 * state-vector hot path of guochu/VQC.jl.
 *
 * Each entry point replaces one Julia method of the reference (cited as
 * file:line within the VQC.jl project).  The Julia side binds them with
 * `ccall` (vqc.jl_b200/julia/VQCB200.jl); the Python host mirror binds them
 * with ctypes (vqc.jl_b200/vqcb200/_lib.py).
 *
 * Conventions, identical to the reference:
 *   - qubits are 0-based here (1-based in Julia): qubit q <-> bit q of the
 *     amplitude index, least significant first (statevector.jl:167-176);
 *   - a k-qubit matrix is row-major 2^k x 2^k, complex interleaved (re, im)
 *     FP64; bit b of its row/column index <-> pos[b], in the order given
 *     (QuantumCircuits' ordered_mat is applied inside);
 *   - a density matrix of n qubits is stored as a 2n-qubit vector: bits
 *     0..n-1 index the row, bits n..2n-1 the column (densitymatrix.jl:27-30);
 *   - amplitudes are complex interleaved, FP32 (VQC_C64) or FP64 (VQC_C128);
 *     every norm, inner product, expectation and gradient is accumulated in
 *     FP64 on the device and returned as FP64.
 *
 * Every function returns 0 (VQC_OK) or a negative status; vqc_last_error()
 * gives the message of the last failure on the calling thread.  A handle owns
 * one CUDA stream; calls on one handle are serialised, calls on different
 * handles may run concurrently from different threads.  Calls that return a
 * host value synchronise the handle's stream; the others are asynchronous
 * unless stated.
 */
#ifndef VQC_B200_H
#define VQC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VQC_OK 0
#define VQC_ERR_ARG (-1)         /* bad argument (throw/@assert/ArgumentError in the reference) */
#define VQC_ERR_OOM (-2)         /* device allocation failed */
#define VQC_ERR_CUDA (-3)        /* CUDA runtime error */
#define VQC_ERR_UNSUPPORTED (-4) /* e.g. a >5-qubit gate (generic.jl:37) */
#define VQC_ERR_TIMEOUT (-5)     /* a bounded wait ran out (serving) */
#define VQC_ERR_BUSY (-6)        /* serving: no slot or memory free for the request now */
#define VQC_ERR_CANCELED (-7)    /* serving: the request was cancelled */

#define VQC_C64 0  /* ComplexF32 amplitudes */
#define VQC_C128 1 /* ComplexF64 amplitudes */

typedef struct vqc_state_s* vqc_state;

/* One gate of a circuit: nq positions, its matrix at mats + mat (in doubles). */
typedef struct {
  int32_t nq;
  int32_t pos[5];
  int64_t mat;
} vqc_gate;

/* One circuit parameter of gate `gate`; its matrix at mats + dmat is
 *   kind VQC_PARAM_DERIVATIVE (0): dU/dtheta, or
 *   kind VQC_PARAM_GENERATOR  (1): the gate G that QuantumCircuits'
 *     differentiate(gate) returns, used by the reference as
 *     grad = real(expectation(y_in, G, delta_in)) (circuitdiff.jl:29). */
typedef struct {
  int32_t gate;
  int32_t kind;
  int64_t dmat;
} vqc_param;
#define VQC_PARAM_DERIVATIVE 0
#define VQC_PARAM_GENERATOR 1

/* One Pauli string coeff * prod_q P_q, P_q = I, X, Z, Y for (x_q, z_q) =
 * (0,0), (1,0), (0,1), (1,1): x bit q of xmask, z bit q of zmask. */
typedef struct {
  uint64_t xmask;
  uint64_t zmask;
  double coeff_re;
  double coeff_im;
} vqc_pauli;

const char* vqc_last_error(void);
const char* vqc_version(void);
/* Number of CUDA devices visible, or a negative status. */
int vqc_device_count(void);

/* ---- state vectors: StateVector{T} (statevector.jl:1-21) ------------------ */
/* StateVector(T, n): |0...0> on `device` (statevector.jl:15-21). */
int vqc_state_create(int n, int dtype, int device, vqc_state* out);
int vqc_state_destroy(vqc_state h);
int vqc_state_nqubits(vqc_state h);  /* stored qubits: 2n for a density matrix */
int vqc_state_dtype(vqc_state h);
/* storage(x) copies (statevector.jl:24): bytes must equal 2^nq * amplitude size. */
int vqc_state_upload(vqc_state h, const void* host, size_t bytes);
int vqc_state_download(vqc_state h, void* host, size_t bytes);
/* reset!(x) (statevector.jl:110-114): |0...0>, or |0><0| for a density matrix. */
int vqc_state_reset(vqc_state h);
/* copy(x) (statevector.jl:30): same qubit count; converts FP32 <-> FP64. */
int vqc_state_copy(vqc_state dst, vqc_state src);
/* y <- a x + b y, a and b complex (re, im): the vector update of the Krylov
 * solvers behind ground_state / time_evolution (utility/groundstate.jl:4-25,
 * KrylovKit's eigsolve / exponentiate with the operator's matvec). */
int vqc_state_axpby(vqc_state y, const double* a, vqc_state x, const double* b);
/* The state with qubit q (0-based) fixed at `value` and removed, times
 * `scale`: dst (one qubit fewer) <- scale * <value|_q src.  The collapsed
 * state of measure(psi, q) (measure.jl:38-46) and post_select(psi, q, v)
 * without keep (postselect.jl:37-44), scale = 1/sqrt(probability). */
int vqc_state_take_qubit(vqc_state src, int q, int value, double scale, vqc_state dst);
/* norm(x) (statevector.jl:53), FP64. */
int vqc_state_norm(vqc_state h, double* out);
/* dot(x, y) = <x|y> (statevector.jl:54), FP64; out = (re, im). */
int vqc_state_dot(vqc_state x, vqc_state y, double* out);
/* Block the caller until the handle's queued work is done. */
int vqc_state_sync(vqc_state h);
/* Device pointer of the amplitudes (for interop; owned by the handle). */
void* vqc_state_device_ptr(vqc_state h);
/* The handle's cudaStream_t (for interop and event timing). */
void* vqc_state_stream(vqc_state h);

/* ---- launch profiling (no counterpart in the reference) -------------------
 * vqc_profile_enable(1) clears the records and starts timing every kernel
 * launch with CUDA events on its stream, per kernel class; (0) stops.  Each
 * class reports launches, total device ms and total algorithmic bytes (the
 * bytes the operation must move at minimum). */
int vqc_profile_enable(int on);
int vqc_profile_count(void);
int vqc_profile_get(int i, char* name, int name_len, long long* launches, double* total_ms, double* total_bytes);
/* Total FMA-pipe flops of record i: 2 x the lane operations of the FMA pipe
 * (fused multiply-adds, multiplies, adds) the class's launches execute, for
 * the kernels bound by arithmetic (the tile passes); 0 for the others. */
int vqc_profile_flops(int i, double* total_flops);
/* Index checks of the debug build (libvqcb200_debug.so, compiled with
 * VQC_DEBUG_CHECKS; no counterpart in the reference): the number of device
 * accesses whose index fell outside its buffer since the last reset (each was
 * skipped, not performed), and out[0..3] = (count, source line, index, limit)
 * of the first.  reset != 0 clears the records.  Always 0 in the release
 * build, which performs no checks; vqc_debug_build() tells which is loaded. */
int vqc_debug_status(int reset, long long* out);
int vqc_debug_build(void);
/* Measured peak of the device's FMA pipe in TFLOP/s (2 flops per FMA lane):
 * a calibration kernel of independent FMA chains on every SM, timed with
 * CUDA events.  kind 0: packed two-lane FP32 (fma.rn.f32x2), 1: scalar
 * FP32, 2: FP64.  The compute roofline of the tile passes (no counterpart
 * in the reference). */
int vqc_fma_peak(int device, int kind, double* tflops);

/* ---- gates: apply!(::Gate, ::StateVector) (applygates/generic/generic.jl:6-14,
 *      _apply_gate_threaded2! in threaded_short_range.jl / threaded_long_range.jl,
 *      specialised kernels in the applygates/specific directory) ------------- */
int vqc_apply_gate(vqc_state h, int k, const int* pos, const double* mat);
/* apply!(::QCircuit, state) (generic.jl:26-31).  fuse != 0 plans the gates
 * into shared-memory tile passes (one HBM round trip per pass); fuse == 0
 * applies them one by one, like the reference. */
int vqc_apply_circuit(vqc_state h, const vqc_gate* gates, int ngates, const double* mats, int fuse);

/* ---- expectation (hamiltonian/expecs/expecs.jl:12-78) --------------------- */
/* expectation(H, psi) for a Pauli sum; out = (re, im) in FP64. */
int vqc_expect_pauli(vqc_state psi, const vqc_pauli* terms, int nterms, double* out);
/* expectation(phi, H, psi) = <phi|H|psi> (expecs.jl:45-74, expec_threaded_2.jl). */
int vqc_expect_pauli2(vqc_state phi, vqc_state psi, const vqc_pauli* terms, int nterms, double* out);
/* expectation_value(pos, M, psi[, phi]) for one dense k<=5-qubit key
 * (expecs.jl:85-130); phi may be NULL for the one-state form. */
int vqc_expect_dense(vqc_state phi, vqc_state psi, int k, const int* pos, const double* mat, double* out);

/* ---- H * psi (hamiltonian/apply_qterms/apply_qterms.jl:13-28) ------------- */
/* out = H psi for a Pauli sum (out is overwritten). */
int vqc_apply_pauli(vqc_state psi, vqc_state out, const vqc_pauli* terms, int nterms);
/* out += M psi on pos for one dense key (short_range_threaded.jl:1519-1524). */
int vqc_apply_dense_add(vqc_state psi, vqc_state out, int k, const int* pos, const double* mat);

/* ---- gradients: the Zygote adjoints of *(circuit, psi) (circuitdiff.jl:2-8,
 *      23-32, 61-78) and of expectation(H, psi) (expecdiff.jl:30-33, 68) ------ */
/* Energy and gradient of real(expectation(H, circuit(theta) * psi0)):
 * forward pass, E = <y|H|y>, cotangent (H + H^dagger) y, then the reverse
 * sweep that uncomputes the forward state instead of storing it.  psi0 is not
 * modified.  grads[j] is dE/dtheta_j for params[j] (any order).  energy =
 * (re, im).  Blocks until the result is on the host. */
int vqc_adjoint_grad(vqc_state psi0, const vqc_gate* gates, int ngates, const double* mats,
                     const vqc_param* params, int nparams, const vqc_pauli* terms, int nterms, double* energy,
                     double* grads);
/* The circuit pullback alone (back_propagate, circuitdiff.jl:61-75): given the
 * output state y = circuit * psi0 and the cotangent delta of a real loss,
 * overwrite y with psi0 (uncomputed) and delta with the input cotangent, and
 * return grads[j] = Re <delta_out | dU/dtheta_j | y_in> for params[j]. */
int vqc_circuit_backward(vqc_state y, vqc_state delta, const vqc_gate* gates, int ngates, const double* mats,
                         const vqc_param* params, int nparams, double* grads);

/* ---- density matrices (densitymatrix.jl, generic.jl:16-24, 54-64,
 *      ptrace.jl:4-53, measure.jl:69-81) ------------------------------------ */
/* DensityMatrix(T, n): |0><0|, stored as a 2n-qubit vector (4^n amplitudes). */
int vqc_dm_create(int n, int dtype, int device, vqc_state* out);
int vqc_dm_nqubits(vqc_state rho);
/* DensityMatrix(psi) = |psi><psi| (densitymatrix.jl:27); psi has n qubits. */
int vqc_dm_from_state(vqc_state rho, vqc_state psi);
/* apply!(::Gate, ::DensityMatrix): rho <- U rho U^dagger.  The reference runs
 * U on the row qubits and conj(U) on the column qubits in two passes; here
 * both act in one pass. */
int vqc_dm_apply_gate(vqc_state rho, int k, const int* pos, const double* mat);
int vqc_dm_apply_circuit(vqc_state rho, const vqc_gate* gates, int ngates, const double* mats, int fuse);
/* partial_tr(rho, sites): out (host) receives the 2^(n-m) x 2^(n-m) result,
 * column-major, complex FP64 interleaved; the kept qubits keep their order. */
int vqc_dm_ptrace(vqc_state rho, int nsites, const int* sites, double* out);
/* real(diag(rho)): out (host) receives 2^n FP64 probabilities. */
int vqc_dm_probs(vqc_state rho, double* out);
/* tr(rho) (densitymatrix.jl:58), FP64 (re, im). */
int vqc_dm_trace(vqc_state rho, double* out);
/* apply!(::QuantumMap, ::DensityMatrix) (applygates/apply_qmaps.jl:5-14),
 * apply_dagger! (:21-30), apply_inverse! (:36-45): rho <- sum_i K_i rho K_i^dagger
 * for the nkraus Kraus operators K_i (2^k x 2^k, row-major, complex FP64
 * interleaved, index bit b <-> pos[b], like gates), applied as the channel's
 * supermatrix on (pos, pos + n) (apply_qmaps.jl:67-77).  mode 0 = apply,
 * 1 = the supermatrix's adjoint, 2 = its inverse.  k = 1 or 2 (the
 * supermatrix is a 2k-qubit gate; the reference's gate kernels stop at 5). */
int vqc_dm_apply_channel(vqc_state rho, int k, const int* pos, int nkraus, const double* kraus, int mode);
/* expectation(x::DensityMatrix, m::Gate, y::DensityMatrix) of the density-
 * matrix pullback (circuitdiff.jl:35-40): out = tr(op(a) M op(b)), FP64
 * (re, im), with M the k-qubit matrix (row-major, index bit b <-> pos[b])
 * acting on the row qubits (left multiplication) and op(x) = x, or x^dagger
 * when dag_x != 0.  The reference's form is dag_a = dag_b = 0. */
int vqc_dm_trace_prod(vqc_state a, int dag_a, vqc_state b, int dag_b, int k, const int* pos, const double* mat,
                      double* out);
/* expectation(::QubitsOperator, ::DensityMatrix) = tr(H rho)
 * (hamiltonian/expecs_dm/expecs_dm.jl:19-30), FP64 (re, im). */
int vqc_dm_expect_pauli(vqc_state rho, const vqc_pauli* terms, int nterms, double* out);

/* ---- allocation-free expectation (no counterpart in the reference) ------
 * For callers that cannot allocate device memory (a fixed arena handed over
 * at start-up, no cudaMalloc/cudaFree afterwards): expectation(H, psi) of a
 * state in the caller's own device buffer `state` (2^nqubits amplitudes of
 * `dtype`, device memory of the current device, else VQC_ERR_ARG), on
 * `stream` (a cudaStream_t, or NULL for the default stream); out = (re, im)
 * in FP64, the quantity vqc_expect_pauli computes, within rounding: this entry
 * point runs the one-amplitude-per-thread Pauli kernel on a reduction grid of
 * at most 296 blocks (its partial sums must fit the static array), so it is
 * slower than vqc_expect_pauli on large states and sums in another order.
 * Host tables live in thread-local storage, not on the caller's stack.  All scratch lives in one static device array of the
 * library (218,112 bytes per GPU that loads the library, held until exit);
 * at most 1024 Pauli terms per call (more: VQC_ERR_ARG).  The first call on a
 * device looks up the array's device address; make that first call before any
 * stream capture.  Calls share the array: calls that overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller.
 * Blocks until the result is on the host. */
int vqc_expect_pauli_noalloc(const void* state, int nqubits, int dtype, const vqc_pauli* terms, int nterms,
                             void* stream, double* out);

/* ---- serving: continuous batching of many circuits on one GPU (no
 *      counterpart in the reference, which evaluates one circuit per call) ----
 * A server owns one GPU stream, a worker thread and `planner_threads`
 * planning threads.  Requests start from |0...0>, run their circuit, and
 * return expectation(H, circuit * psi0) and, if want_grad, its gradient (the
 * same quantities as vqc_adjoint_grad).  Admission is by device memory: a
 * request is admitted when its states, descriptors and scratch fit
 * `memory_bytes` and fewer than `max_active` requests run.  Every loop
 * iteration advances every admitted request by one step, the steps of a kind
 * in few launches (FP32 passes on run-time compiled kernels, one launch per
 * pass structure); requests arriving meanwhile join at the next iteration.  A
 * request's result does not depend on the requests it is batched with. */
typedef struct vqc_server_s* vqc_server;
int vqc_serve_open(int device, int dtype, size_t memory_bytes, int max_active, int planner_threads,
                   vqc_server* out);
/* Queues one request (inputs are copied).  grads_out (nparams doubles) must
 * stay valid until vqc_serve_poll / vqc_serve_wait has reported the request's
 * outcome (a result, an error, or VQC_ERR_CANCELED).  Gates must have at
 * most two target qubits (controls read off the matrix), 9..40 qubits.  A
 * request with a non-finite matrix entry or Pauli coefficient is rejected
 * here (VQC_ERR_ARG) and never reaches the device. */
int vqc_serve_submit(vqc_server s, int nqubits, const vqc_gate* gates, int ngates, const double* mats,
                     const vqc_param* params, int nparams, const vqc_pauli* terms, int nterms, int want_grad,
                     double* grads_out, int64_t* ticket);
/* 0: not finished; 1: finished (energy and latency_s = completion - submission
 * filled, the ticket is released); negative: the request failed. */
int vqc_serve_poll(vqc_server s, int64_t ticket, double* energy, double* latency_s);
/* As vqc_serve_poll but waits up to timeout_ms (then VQC_ERR_TIMEOUT). */
int vqc_serve_wait(vqc_server s, int64_t ticket, int timeout_ms, double* energy, double* latency_s);
/* Cancels a request: one still queued or planned is dropped at once, one
 * running is retired at the worker's next iteration (its device memory goes
 * back to the budget, its partial results are discarded).  Returns 1 when the
 * cancellation was registered before the request finished -- poll / wait then
 * report VQC_ERR_CANCELED and release the ticket -- 0 when it had already
 * finished (its result stays available), negative for an unknown ticket.
 * Requests batched with it are not affected. */
int vqc_serve_cancel(vqc_server s, int64_t ticket);
/* out[0..6]: completed, loop iterations, launches, request-steps launched,
 * device bytes admitted, requests running, requests waiting. */
int vqc_serve_stats(vqc_server s, long long* out);
/* out[0..5] (seconds): mean and max planning time, mean and max wait for
 * admission, mean and max time from admission to completion. */
int vqc_serve_timing(vqc_server s, double* out);
/* out[0..3]: over the loop iterations that launched work, the summed host time
 * building and enqueueing the batched launches, the summed wait for the device,
 * the summed host time retiring finished requests (seconds), and the number of
 * such iterations.  Diagnostic; the reference has no serving loop. */
int vqc_serve_loop_timing(vqc_server s, double* out);
int vqc_serve_close(vqc_server s);

#ifdef __cplusplus
}
#endif
#endif /* VQC_B200_H */
