/*
 * qclab_b200.h -- C ABI of the B200 state-vector backend for QCLAB++.
 *
 * Every entry point is plain C: integers, doubles, raw pointers and sizes.
 * Every entry point returns a qsv_status (0 = success) and never aborts;
 * qsv_last_error() returns a message for the last failure on the calling
 * thread.  All device work is issued on the state's CUDA stream (the legacy
 * default stream unless qsv_set_stream was called); calls that return host
 * values (downloads, reductions) synchronise that stream.  Calls on two
 * states with different streams order themselves on the device: the work
 * starts after both streams' earlier work, and later work on either stream
 * starts after it (CUDA events, no host synchronisation).
 *
 * Conventions follow QCLAB++ exactly:
 *   - qubit q of an n-qubit register is bit (n-1-q) of the amplitude index
 *     (qubit 0 is the most significant bit)      [src/qgates/apply.hpp:227-238]
 *   - an op is 'N' (NoTrans), 'T' (Trans) or 'C' (ConjTrans) and is applied
 *     to every gate; for 'T'/'C' the gate list runs in reverse order
 *                                               [include/qclab/QCircuit.hpp:130-143]
 *   - rotations carry cos/sin of theta/2 (QRotation), Phase and CPhase carry
 *     cos/sin of theta (QAngle)     [include/qclab/QRotation.hpp:44-66,
 *                                    include/qclab/QAngle.hpp:30-48]
 *   - dense matrices are column-major, complex entries stored as (re, im)
 *                                    [include/qclab/dense/SquareMatrix.hpp:57-78]
 */
#ifndef QCLAB_B200_H
#define QCLAB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QSV_ABI_VERSION 1

typedef enum qsv_status {
  QSV_SUCCESS             = 0,
  QSV_ERROR_INVALID_VALUE = 1,  /* null pointer, unknown enum, bad op char   */
  QSV_ERROR_QUBIT         = 2,  /* qubit outside [0,nbQubits) or repeated    */
  QSV_ERROR_SIZE          = 3,  /* byte count or problem size out of range   */
  QSV_ERROR_CUDA          = 4,  /* CUDA runtime failure (see qsv_last_error) */
  QSV_ERROR_OUT_OF_MEMORY = 5,  /* device allocation failed                  */
  QSV_ERROR_DTYPE         = 6,  /* gate not defined for a real element type  */
  QSV_ERROR_TIMEOUT       = 7,  /* a bounded device-side wait expired        */
  QSV_ERROR_NOT_SUPPORTED = 8
} qsv_status;

/* Element type of a state vector (the QCLAB++ template parameter T). */
typedef enum qsv_dtype {
  QSV_C64  = 0,   /* std::complex<float>  */
  QSV_C128 = 1,   /* std::complex<double> */
  QSV_F32  = 2,   /* float                */
  QSV_F64  = 3    /* double               */
} qsv_dtype;

/* Gate kinds: one per QCLAB++ gate class on the state-vector path, plus the
 * generic matrix gates (U2/U3/MatrixGate) that QCLAB++ lacks.               */
typedef enum qsv_gate_kind {
  QSV_IDENTITY      = 0,   /* qgates/Identity                                 */
  QSV_HADAMARD      = 1,   /* qgates/Hadamard                                 */
  QSV_PAULI_X       = 2,   /* qgates/PauliX                                   */
  QSV_PAULI_Y       = 3,   /* qgates/PauliY                                   */
  QSV_PAULI_Z       = 4,   /* qgates/PauliZ                                   */
  QSV_ROTATION_X    = 5,   /* qgates/RotationX   (cos,sin of theta/2)         */
  QSV_ROTATION_Y    = 6,   /* qgates/RotationY   (cos,sin of theta/2)         */
  QSV_ROTATION_Z    = 7,   /* qgates/RotationZ   (cos,sin of theta/2)         */
  QSV_PHASE         = 8,   /* qgates/Phase       (cos,sin of theta)           */
  QSV_PHASE45       = 9,   /* qgates/Phase45 (T gate)                         */
  QSV_PHASE90       = 10,  /* qgates/Phase90 (S gate)                         */
  QSV_MATRIX1       = 11,  /* QGate1 / PointerGate1 / U2 / U3: matrix[0..7]   */
  QSV_CX            = 12,  /* qgates/CX (= CNOT)                              */
  QSV_CY            = 13,  /* qgates/CY                                       */
  QSV_CZ            = 14,  /* qgates/CZ                                       */
  QSV_CPHASE        = 15,  /* qgates/CPhase      (cos,sin of theta)           */
  QSV_CROTATION_X   = 16,  /* qgates/CRotationX  (cos,sin of theta/2)         */
  QSV_CROTATION_Y   = 17,  /* qgates/CRotationY  (cos,sin of theta/2)         */
  QSV_CROTATION_Z   = 18,  /* qgates/CRotationZ  (cos,sin of theta/2)         */
  QSV_CONTROLLED1   = 19,  /* QControlledGate2 with any 2x2 target matrix     */
  QSV_SWAP          = 20,  /* qgates/SWAP                                     */
  QSV_ISWAP         = 21,  /* qgates/iSWAP                                    */
  QSV_ROTATION_XX   = 22,  /* qgates/RotationXX  (cos,sin of theta/2)         */
  QSV_ROTATION_YY   = 23,  /* qgates/RotationYY  (cos,sin of theta/2)         */
  QSV_ROTATION_ZZ   = 24,  /* qgates/RotationZZ  (cos,sin of theta/2)         */
  QSV_MATRIX2       = 25,  /* QGate2 / PointerGate2 / MatrixGate2: 4x4        */
  QSV_NUM_GATE_KINDS = 26
} qsv_gate_kind;

/*
 * One gate record (the flat form of a qclab::QObject<T> gate).
 *   1-qubit kinds     : qubit0 = the qubit.
 *   controlled kinds  : qubit0 = control, qubit1 = target, control_state 0/1.
 *   SWAP/iSWAP/RXX/RYY/RZZ : qubit0, qubit1 in any order (sorted as QCLAB++
 *                       does, include/qclab/qgates/QRotationGate2.hpp:142-147).
 *   MATRIX2           : 4x4 in the basis |qubit0 qubit1>, qubit0 the leading
 *                       tensor factor (either order of qubit0/qubit1 allowed).
 *   param             : index of the trainable angle this gate depends on
 *                       (adjoint gradients), or -1.
 */
typedef struct qsv_gate {
  int32_t kind;
  int32_t qubit0;
  int32_t qubit1;
  int32_t control_state;
  double  cos;
  double  sin;
  double  matrix[32];
  int32_t param;
  int32_t reserved;
} qsv_gate;

typedef struct qsv_state_s* qsv_state;

/* ---- library ------------------------------------------------------------ */
int         qsv_abi_version(void);
const char* qsv_last_error(void);
const char* qsv_status_string(qsv_status status);
/* number of kernel launches this library has issued on the calling thread */
uint64_t    qsv_launch_count(void);
/* of those, stage launches whose tiles moved between global and shared
 * memory by TMA (cp.async.bulk.tensor)                                     */
uint64_t    qsv_tma_launch_count(void);

/* ---- state vectors ------------------------------------------------------ */
/* Allocates a 2^nbQubits state on the current device, set to |0...0>.
 * Replaces std::vector<T>(N) + psi[0]=1 of test/timings/run.hpp:50-52.     */
qsv_status qsv_create(int nbQubits, qsv_dtype dtype, qsv_state* out);
/* Non-owning view of caller-owned device memory (QCLAB++'s device T*,
 * QCircuit::simulate_device, include/qclab/QCircuit.hpp:170-172).          */
qsv_status qsv_wrap(int nbQubits, qsv_dtype dtype, void* device_ptr,
                    qsv_state* out);
qsv_status qsv_destroy(qsv_state state);
qsv_status qsv_set_stream(qsv_state state, void* cuda_stream);
qsv_status qsv_info(qsv_state state, int* nbQubits, qsv_dtype* dtype,
                    void** device_ptr);
qsv_status qsv_upload(qsv_state state, const void* host, size_t bytes);
qsv_status qsv_download(qsv_state state, void* host, size_t bytes);
/* dst <- src (same size and dtype), issued on dst's stream. */
qsv_status qsv_copy(qsv_state dst, qsv_state src);
/* |index> (a computational basis state, big-endian qubit order). */
qsv_status qsv_set_basis(qsv_state state, uint64_t index);
qsv_status qsv_synchronize(qsv_state state);

/* ---- gate application --------------------------------------------------- */
/* Reference-exact path: one kernel per gate, with the operation order of the
 * reference lambdas and no FMA contraction, so results are bitwise equal to
 * QCLAB++'s CPU apply.  Replaces QObject<T>::apply(Op, nbQubits, vector,
 * offset) (include/qclab/QObject.hpp:52-53) and the QCircuit gate loop
 * (include/qclab/QCircuit.hpp:130-143).                                     */
qsv_status qsv_apply(qsv_state state, const qsv_gate* gates, size_t nGates,
                     char op, int offset);

/* Options of the fused sweep. Zero-initialised fields pick tuned defaults. */
typedef struct qsv_fuse_opts {
  int tile_bits;     /* m: amplitudes per shared-memory tile = 2^m           */
  int low_bits;      /* L: contiguous low bits always in the tile            */
  int reg_bits;      /* k: qubits per register block inside a tile           */
  int max_stage_gates;
  int profile;       /* 1: time every stage with CUDA events (see below)   */
  int engine;        /* complex single-vector sweeps:
                        0 (default) = 5 for complex<float>, 2 for
                        complex<double>;
                        1 = sparse register passes on the CUDA cores;
                        2 = every register pass of 3 tile bits multiplied
                        out into an 8x8 complex matrix in FP64 and applied
                        on the FP64 tensor cores (mma.sync f64),
                        complex<float> states rounded once per pass;
                        3 = complex<float>: TF32 three-term split on tcgen05
                        with the state rows in tensor memory (tiles of
                        2^10 .. 2^13 amplitudes, else as 4);
                        4 = complex<float>: TF32 three-term split on
                        mma.sync (the TF32 engines' FP32 accumulation
                        truncates: the norm shrinks by about 1e-7 per pass);
                        5 = gate-specialised register passes: every gate is
                        one op whose register positions are compile-time,
                        one-qubit gates factored to two multiply-adds per
                        component with their scalar applied once per stage,
                        in the state's precision (reg_bits 4, or 5 for
                        complex<float>, the default there).
                        Two-vector (adjoint) sweeps use 5 unless 1 is
                        asked for.                                           */
  int ctas_per_sm;   /* engine 5: resident CTAs per SM the stage kernel is
                        built for (0 = default; 2 or 3)                    */
  int tile_copy;     /* engine 5: how tiles move between global and shared
                        memory: 0 (default) = TMA (cp.async.bulk.tensor,
                        one thread per CTA, 128-byte swizzle) wherever the
                        stage's tile fits a 5-D tensor map, else 1;
                        1 = 16-byte cp.async by every thread              */
} qsv_fuse_opts;

/* Fused path: the gate list is planned into stages; each stage streams the
 * state through shared memory once and applies all of its gates there.
 * Within 1e-12 (complex<double>) of qsv_apply, not bitwise.  Gates are
 * lowered and multiplied out in FP64 for every element type, so for a
 * complex<float> state the fused result is closer to the exact circuit than
 * the reference's float arithmetic (qsv_apply reproduces the latter).     */
qsv_status qsv_apply_fused(qsv_state state, const qsv_gate* gates,
                           size_t nGates, char op, int offset,
                           const qsv_fuse_opts* opts);

/* Per-stage kernel durations (ms, CUDA events on the state's stream) of the
 * last qsv_apply_fused call on this thread that ran with opts->profile = 1.
 * Synchronises nothing; the profiled call already waited for its events. */
qsv_status qsv_last_stage_times(float* ms, int capacity, int* count);

/* Plan statistics for a gate list (no device work): number of stages and
 * of ops per stage -- gates for the sparse engine (opts->engine = 1), one
 * dense matrix per register pass for the tensor-core engine.  stage_gates
 * may be NULL.  With opts->low_bits unset, the tensor-core engine plans
 * several low-bit counts and reports the plan it would run (the one with
 * the least passes + a per-element-size weight of stages).                */
qsv_status qsv_plan_stats(int nbQubits, qsv_dtype dtype, const qsv_gate* gates,
                          size_t nGates, char op, int offset,
                          const qsv_fuse_opts* opts, int* nStages,
                          int* stage_gates, int capacity);
/* Host only (new): totals of the same plan -- stages, register passes (one
 * shared-memory round trip of a tile each) and ops. */
qsv_status qsv_plan_passes(int nbQubits, qsv_dtype dtype, const qsv_gate* gates,
                           size_t nGates, char op, int offset,
                           const qsv_fuse_opts* opts, int* nStages, int* nPasses,
                           int* nOps);

/* ---- FP64 reductions (new: QCLAB++ has no observables) -------------------
 * All sums accumulate in double precision whatever the state's dtype, with
 * a deterministic two-stage reduction (per-CTA partials, then one fixed-order
 * pass), so repeated calls give identical bits.
 *
 * Observables are sums of Pauli strings: `paulis` holds nTerms strings of
 * nbQubits characters from {I,X,Y,Z}; character q of a term is the Pauli on
 * qubit q (qubit 0 first, the QCLAB++ order).  coefs[t] is its real weight. */

/* <psi|psi> */
qsv_status qsv_norm2(qsv_state state, double* out);
/* psi /= sqrt(<psi|psi>) with the norm formed in FP64 (removes the norm
 * drift that rounding leaves in long complex<float> sweeps); *norm2_out
 * (may be NULL) receives <psi|psi> before the scaling. */
qsv_status qsv_normalize(qsv_state state, double* norm2_out);
/* <a|b> as (re, im); a and b must have the same size and dtype. */
qsv_status qsv_inner(qsv_state a, qsv_state b, double* out_re_im);
/* Compares two states of the same size, possibly of different dtypes (the
 * precision study: a complex<float> state against a complex<double> one):
 * out[0], out[1] = <a|b> (re, im) and out[2] = max_j |a_j - b_j|, all in
 * FP64.  Infidelity = 1 - |<a|b>|^2 for normalised states.               */
qsv_status qsv_compare(qsv_state a, qsv_state b, double* out3);
/* <psi|H|psi> for H = sum_t coefs[t] * paulis[t]. */
qsv_status qsv_expectation(qsv_state state, const char* paulis,
                           const double* coefs, size_t nTerms, double* out);
/* <psi|H|psi> like qsv_expectation, for callers that must not allocate
 * device memory -- e.g. a host program or framework that has already
 * reserved the GPU's memory for its own pool allocator (a cudaMalloc from
 * this library would fail or fragment that pool), or a tight optimisation
 * loop that cannot afford cudaMalloc/cudaFree, which synchronise the
 * device.  No counterpart in the reference (QCLAB++ has no observables).
 *   state       : caller-owned device array of 2^nbQubits elements of dtype,
 *                 on the current device (QSV_ERROR_INVALID_VALUE otherwise).
 *   cuda_stream : stream to run on (NULL = legacy default stream); the call
 *                 synchronises it before returning.
 * Calls no cudaMalloc/cudaFree: its work memory is a fixed 1 MiB array
 * inside the library, held by every GPU that loads the library until the
 * process exits.  An observable whose term table, run offsets and partial
 * sums need more than 1 MiB is rejected with QSV_ERROR_SIZE (use
 * qsv_expectation).  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress, with the device current); make that
 * first call before any stream capture.  All calls share the array: calls
 * that overlap on the GPU (other streams, other host threads) race.       */
qsv_status qsv_expectation_noalloc(const void* state, int nbQubits,
                                   qsv_dtype dtype, void* cuda_stream,
                                   const char* paulis, const double* coefs,
                                   size_t nTerms, double* out);
/* dst = H src (dst != src, same size and dtype; products formed in FP64),
 * issued on src's stream. */
qsv_status qsv_apply_observable(qsv_state dst, qsv_state src,
                                const char* paulis, const double* coefs,
                                size_t nTerms);

/* ---- adjoint gradient (new: QCLAB++ has no differentiation) ---------------
 * E(theta) = <psi|U^+ H U|psi> and dE/dtheta_p for every trainable angle:
 * gates with param = p >= 0 (RotationX/Y/Z, RotationXX/YY/ZZ, CRotationX/Y/Z,
 * Phase, CPhase; theta is the full angle of QRotation(theta)/QAngle(theta))
 * contribute to grads[p]; gates sharing p add up.  One forward fused sweep,
 * then one backward fused sweep that uncomputes psi and lambda = H psi with
 * the inverse gates (no stored intermediate states).
 *   state : psi on input; on return it holds psi again, recomputed by the
 *           inverse gates (equal to the input up to rounding).
 *   grads : nParams doubles (overwritten).     expval: E (may be NULL).
 * Uses one extra state-sized work vector owned by the state object.        */
qsv_status qsv_adjoint_gradient(qsv_state state, const qsv_gate* gates,
                                size_t nGates, const char* paulis,
                                const double* coefs, size_t nTerms,
                                double* grads, int nParams, double* expval);

/* ---- batched variational sweeps (new: no reference counterpart) ------------
 * Many independent circuits, each with its own qubit count (5..30), gate
 * list and Pauli-sum observable: energy E_c = <psi_c|H_c|psi_c> from |0...0>
 * and the full adjoint gradient dE_c/dtheta_p of every circuit, computed by
 * ONE persistent kernel launch (largest circuits first; a circuit whose two
 * work vectors fit a CTA's shared memory runs on one CTA and never touches
 * HBM, a larger one on a team of CTAs that share its tiles stage by stage)
 * that qsv_batch_run can capture in a CUDA graph.  Team barriers wait a
 * bounded time; if one gives up, qsv_batch_results returns
 * QSV_ERROR_TIMEOUT.
 *   gates + gate_offsets[c..c+1]     : circuit c's records (param >= 0 marks
 *                                      a trainable angle, < nParams[c])
 *   paulis/coefs + term_offsets[c..] : circuit c's terms (nbQubits[c] chars
 *                                      each, strings back to back)
 * Results: energies[nCircuits], gradients concatenated in circuit order.  */
typedef struct qsv_batch_s* qsv_batch;
typedef struct qsv_batch_opts {
  int tile_bits;     /* 2^m amplitudes per shared-memory tile (0 = default) */
  int low_bits;      /* contiguous low bits of a tile (0 = default)          */
  int ctas_per_sm;   /* cap on resident CTAs per SM (0 = occupancy limit)   */
  int max_team;      /* most CTAs sharing one circuit larger than a tile
                        (0 = 16; 1 = one CTA per circuit)                    */
  int reserved[4];
} qsv_batch_opts;
qsv_status qsv_batch_create(qsv_dtype dtype, int nCircuits, const int* nbQubits,
                            const qsv_gate* gates, const size_t* gate_offsets,
                            const char* paulis, const double* coefs,
                            const size_t* term_offsets, const int* nParams,
                            const qsv_batch_opts* opts, qsv_batch* out);
/* One launch of the whole batch on cuda_stream; use_graph != 0 captures it
 * (results reset + persistent kernel) in a CUDA graph on first use and
 * replays the graph afterwards. */
qsv_status qsv_batch_run(qsv_batch batch, void* cuda_stream, int use_graph);
qsv_status qsv_batch_results(qsv_batch batch, void* cuda_stream,
                             double* energies, double* gradients);
qsv_status qsv_batch_info(qsv_batch batch, int* blocks, int* threads,
                          int* tile_bits, size_t* workspace_bytes);
/* Work of one launch, from the plan: global_bytes = tile traffic of the
 * circuits larger than a tile (each stage reads and writes its vectors once;
 * circuits that fit a tile stay in shared memory and move none);
 * amplitude_updates = sum over circuits of 2^n x (forward gates + 2 x
 * backward gates).  Either pointer may be NULL. */
qsv_status qsv_batch_work(qsv_batch batch, double* global_bytes,
                          double* amplitude_updates);
qsv_status qsv_batch_destroy(qsv_batch batch);

/* ---- device probe (new) --------------------------------------------------
 * FP64 tensor-core throughput of the current device in TFLOP/s (mma.sync
 * m8n8k4 f64, a few ms): the peak the fused complex sweep is measured
 * against.  Allocates and frees a small buffer.                            */
qsv_status qsv_fp64_mma_peak(double* tflops);

/* ---- unitaries ---------------------------------------------------------------
 * A 2^n x 2^n matrix lives on the device in a state object of 2n qubits
 * (qsv_create(2n, ...)) holding its entries column-major -- (r, c) at
 * r + c 2^n, the layout of qclab::dense::SquareMatrix.  Gates address the n
 * matrix qubits.                                                             */
/* qclab::dense::eye: the identity, the start of QCircuit::matrix()
 * (include/qclab/QCircuit.hpp:120-126).  QSV_ERROR_SIZE for an odd count. */
qsv_status qsv_set_identity(qsv_state matrix);
/* QObject<T>::apply(Side side, Op op, nbQubits, SquareMatrix<T>&, offset)
 * for a gate list in circuit order (include/qclab/QCircuit.hpp:176-204;
 * per gate src/qgates/QGate1.cpp:27-80, QGate2.cpp, QControlledGate2.cpp):
 * side 'R' gives matrix <- op(U) matrix, side 'L' matrix <- matrix op(U).
 * fused != 0 runs the fused stage sweep, else the per-gate kernels.       */
qsv_status qsv_apply_matrix(qsv_state matrix, const qsv_gate* gates, size_t nGates,
                            char side, char op, int offset, int fused);
/* qclab::nrmF (include/qclab/QCircuit.hpp:407-430): scale * sqrt(sum
 * |(a - b) / scale|^2) with scale = max |a - b| (1 if zero), in FP64, for
 * two objects of the same size (any element types).                      */
qsv_status qsv_nrmF(qsv_state a, qsv_state b, double* out);

/* ---- OpenQASM front end ----------------------------------------------------
 * Parses OpenQASM text exactly as QCLAB++'s QASMFile does
 * (include/qclab/io/QASMFile.hpp:42-167, src/io/QASMFile.cpp:16-53): gates
 * h x y z rx ry rz p cx cy cz swap on one qreg, other commands skipped,
 * angles read with stof/stod in dtype's precision.  Writes up to capacity
 * records to gates (may be NULL to query), *count = gates parsed,
 * *nbQubits = register size.  A command the reference cannot parse (e.g. an
 * angle "pi/2") returns QSV_ERROR_INVALID_VALUE with the gates read so far,
 * as the reference keeps them.                                             */
qsv_status qsv_parse_qasm(const char* text, qsv_dtype dtype, qsv_gate* gates,
                          size_t capacity, size_t* count, int* nbQubits);

/* Host-buffer convenience, the drop-in for QCircuit<T>::simulate(vector)
 * (include/qclab/QCircuit.hpp:164-166): copies `host` (2^nbQubits elements
 * of dtype) to the device, applies the gate list with `op`, copies back.
 * fused != 0 selects qsv_apply_fused.                                      */
qsv_status qsv_apply_host(int nbQubits, qsv_dtype dtype, void* host,
                          const qsv_gate* gates, size_t nGates, char op,
                          int offset, int fused);

#ifdef __cplusplus
}
#endif

#endif /* QCLAB_B200_H */
