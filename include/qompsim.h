/*
 * qompsim.h -- C ABI of the B200 compressed state-vector engine.
 *
 * Plain C: opaque handles, pointers and sizes, integer status codes.  No C++
 * type and no exception crosses this boundary.  Each entry point names the
 * reference interface it replaces (paths are relative to the reference
 * project, FujitsuResearch/Compression-based-State-Vector-Simulator).
 *
 * Two handle types:
 *   qs_state  -- the block-wise compressed state (CompressedQuantumState,
 *                src/cppsim/compressed_state.hpp:9).  The compressed store
 *                lives in device memory (HBM) for the whole life of the
 *                handle (its payload in mapped host memory with
 *                QS_FLAG_HOST_STORE); the reference kept it in host malloc
 *                buffers and moved every group over PCIe each stage
 *                (src/cppsim/compressed_state_cuda.cu:209-223, 343-370).
 *   qs_dense  -- an uncompressed state vector in device memory (QuantumState,
 *                src/cppsim/state.hpp:445-1045, updated gate by gate through
 *                QuantumCircuit::update_quantum_state, src/cppsim/circuit.cpp:23-34).
 *
 * Threading: a handle is not re-entrant; use one handle per host thread.
 * Handles on different threads may run concurrently (the per-kernel launch
 * settings they share are only ever raised, under a lock).
 * All device work of a handle is ordered on one CUDA stream (qs_set_stream,
 * default: the legacy default stream).  Calls that return host data
 * synchronise that stream.  qs_apply_circuit reads its per-stage flags and
 * final counters through mapped host memory written by its own kernels, not
 * through copies, so on its own stream it never waits for another stream's
 * host transfers (a store export on another handle, for example).
 */
#ifndef QOMPSIM_H
#define QOMPSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum qs_status {
    QS_OK = 0,
    QS_ERR_ARG = 1,              /* invalid argument (sizes, indices, bounds)          */
    QS_ERR_CUDA = 2,             /* a CUDA runtime call failed                          */
    QS_ERR_CAPACITY = 3,         /* compressed store does not fit its arenas            */
    QS_ERR_UNSUPPORTED_GATE = 4, /* gate with >2 qubits, FusedSWAP (needs MPI ranks)    */
    QS_ERR_TIMEOUT = 5,          /* a bounded device wait gave up                       */
    QS_ERR_CORRUPT = 6,          /* imported store failed its length/header checks      */
    QS_ERR_STATE = 7,            /* call out of order (e.g. apply before registration)  */
    QS_ERR_NOMEM = 8,            /* host allocation failed                              */
    QS_ERR_DOMAIN = 9            /* no finite positive probability mass to sample from  */
} qs_status;

typedef enum qs_dtype {
    QS_COMPLEX128 = 0,  /* amplitudes and gate arithmetic in FP64             */
    QS_COMPLEX64 = 1    /* amplitudes and gate arithmetic in FP32; FP64 norms */
} qs_dtype;

/* Flags of qs_create. */
#define QS_FLAG_EXACT_ZERO_TEST 0x1u /* the reference GPU build's exact |a|^2 != 0 test
                                        (cuda_complex_helper.cuh:96-106) for blocks that were
                                        zero before a stage.  Default: the block stays zero
                                        when every amplitude quantises to code 0, i.e. |re|,
                                        |im| <= 2^-(L+1) -- the CPU build's threshold test
                                        (compressed_state.hpp:939-951) at the codec's
                                        resolution, immune to FMA rounding residues */
#define QS_FLAG_REFERENCE_CONTROLS 0x2u /* reproduce the reference dispatch: controls are
                                        honoured for "CNOT" only and 2x2 / 4x4 matrices are
                                        applied uncontrolled, 4x4 bit0 on the lower target
                                        (compressed_state.hpp:998-1008, compressed_state_cuda.cu:632-642) */
#define QS_FLAG_QUIET 0x4u           /* no progress prints on stdout */
#define QS_FLAG_PROFILE 0x8u         /* time every fused pass with CUDA events (qs_stats.kernel_ms) */
#define QS_FLAG_HOST_STORE 0x10u     /* spill tier: the compressed payload arenas live in pinned,
                                        device-mapped host memory (a quarter of the host's free
                                        memory each unless QOMPSIM_ARENA_BYTES says otherwise) and
                                        the passes stream them over the bus; chunk headers, masks
                                        and counters stay in HBM.  Also set by QOMPSIM_HOST_STORE=1.
                                        The reference keeps its blocks in host memory
                                        (compressed_state_cuda.cu:343) */

/* One gate as the reference's partition_and_register_circuit binding hands
 * it to the engine: to_matrix_gate(gate) with the original name kept
 * (python/cppsim_wrapper.cpp:465-482). */
typedef struct qs_gate {
    char name[24];               /* "CNOT", "DenseMatrix", "H", ... ; "FusedSWAP" is rejected */
    uint32_t ntargets;           /* 1 or 2                                                    */
    uint32_t ncontrols;          /* 0..2 (targets + controls <= 2 unless REFERENCE_CONTROLS)   */
    uint32_t targets[2];         /* matrix index bit i <-> targets[i]                          */
    uint32_t controls[2];
    uint32_t control_values[2];
    double matrix[32];           /* row-major 2^ntargets x 2^ntargets, interleaved re, im      */
} qs_gate;

typedef struct qs_state qs_state;
typedef struct qs_dense qs_dense;

/* Codec / engine statistics of the last qs_apply_circuit. */
typedef struct qs_stats {
    uint64_t stages;             /* reference stages executed                          */
    uint64_t passes;             /* device passes, tile passes + perm_passes (>= 1 per stage) */
    uint64_t tiles;              /* tiles processed (tile passes)                      */
    uint64_t bytes_read;         /* compressed payload + chunk headers read (tile passes) */
    uint64_t bytes_written;      /* compressed payload + chunk headers written (tile passes) */
    uint64_t amp_gate_updates;   /* sum over stages of gates(s) * amplitudes in active groups(s) */
    double kernel_ms;            /* device time of the fused tile passes alone (QS_FLAG_PROFILE),
                                    else equal to apply_ms                             */
    double apply_ms;             /* device time of qs_apply_circuit end to end          */
    int32_t mantissa_bits;       /* quantiser parameter m (relative step 2^-m)          */
    int32_t linear_exp;          /* quantiser parameter L (absolute step 2^-L)          */
    int32_t chunk_log2;          /* amplitudes per chunk = 2^chunk_log2                 */
    int32_t tile_log2;           /* largest tile = 2^tile_log2 amplitudes               */
    uint64_t sweeps;             /* register sweeps over all passes (plan)              */
    uint64_t ops;                /* gate op records over all passes (plan)              */
    uint64_t perm_passes;        /* passes that only permute chunk headers (SWAP / X on
                                    qubits >= chunk_log2, applied without decoding)     */
    uint64_t perm_bytes;         /* chunk-header bytes read + written by those passes   */
    double perm_ms;              /* their device time (QS_FLAG_PROFILE), else 0         */
    uint64_t code_move_passes;   /* tile passes made only of X / SWAP moves, which carry the
                                    quantised codes through the tile without dequantising */
    uint64_t arena_capacity;     /* bytes of each of the two payload arenas             */
    uint64_t host_store;         /* 1 when the arenas are in host memory (QS_FLAG_HOST_STORE) */
    int64_t merged_from;         /* first stage of the merged tail of the last apply, -1 when none:
                                    once every block is stored, the remaining stages' gates share
                                    passes (no stage boundary can change the mask any more) */
    uint64_t tail_passes;        /* device passes of that merged tail                   */
    double pair_ms;              /* device time (CUDA events) of the launches of the
                                    last qs_apply_pauli_sum / qs_adjoint on this state */
} qs_stats;

/* ---------------------------------------------------------------- errors */

/* Text of the last error of `h`, or of the last failed qs_create /
 * qs_dense_create when h is NULL.  Never NULL. */
const char *qs_last_error(const qs_state *h);
const char *qs_dense_last_error(const qs_dense *h);

/* ------------------------------------------------------ compressed state */

/* CompressedQuantumState(qubit_count, block_size) -- compressed_state.hpp:87-239
 * and initialize_all_blocks (:327-352): block 0 holds |0...0>, all other
 * blocks are zero (not stored).  eps_rel / eps_abs play the role of
 * BITCOMP_REL_EB / BITCOMP_ABS_EB (:128-139); eps_rel must lie in
 * [2^-24, 1).  Requires 4 <= block_size <= n <= 40. */
qs_status qs_create(qs_state **out, uint32_t n, uint32_t block_size, qs_dtype dtype,
                    double eps_rel, double eps_abs, uint32_t flags);

/* ~CompressedQuantumState -- compressed_state.hpp:244-285. */
qs_status qs_destroy(qs_state *h);

/* Order all later device work of h on `cuda_stream` (a cudaStream_t). */
qs_status qs_set_stream(qs_state *h, void *cuda_stream);

/* Copy a gate list in (the gate_list argument of partition_and_register_circuit /
 * register_circuit_stages, compressed_state.hpp:464-474, 673-682). */
qs_status qs_register_gates(qs_state *h, const qs_gate *gates, size_t count);

/* partition_and_register_circuit(gate_list, inner_size, verbose) --
 * compressed_state.hpp:673-726: partition_circuit (:509-583) then
 * make_block_groups (:585-671).  verbose > 0 prints "Circuit Stages: [...]",
 * verbose > 1 also the block groups. */
qs_status qs_partition(qs_state *h, uint32_t inner_size, int verbose);

/* register_circuit_stages(gate_list, stages, block_to_group_list, stage_num_groups)
 * -- compressed_state.hpp:464-474.  stage_gate_ids holds the gate indices of
 * all stages back to back (stage_sizes[s] of them for stage s);
 * block_to_group holds nstages * nblocks group ids. */
qs_status qs_register_stages(qs_state *h, const uint32_t *stage_sizes, size_t nstages,
                             const uint32_t *stage_gate_ids, const uint32_t *block_to_group,
                             const uint32_t *num_groups);

/* partition_circuit + make_block_groups on the host only (no device is
 * touched): the stage plan qs_partition would build for `gates` on an
 * n-qubit state with 2^block_size-amplitude blocks.  Call with NULL outputs
 * to get *nstages; then stage_sizes (nstages), stage_gate_ids (count),
 * block_to_group (nstages * 2^(n-block_size)) and num_groups (nstages),
 * each may be NULL.  Restates compressed_state.hpp:509-671. */
qs_status qs_plan_stages(const qs_gate *gates, size_t count, uint32_t n, uint32_t block_size,
                         uint32_t inner_size, size_t *nstages, uint32_t *stage_sizes,
                         uint32_t *stage_gate_ids, uint32_t *block_to_group, uint32_t *num_groups);

/* Planner introspection (host only; no reference counterpart): the gates of
 * ONE stage as the engine applies them.  SWAP and X gates (and other
 * bit-moving 0/1 permutations) whose qubits are all >= chunk_log2 move whole
 * chunks; the engine folds them into a chunk-index permutation sigma that the
 * stage's last pass applies when it stores the chunks (a stage made only of
 * such gates becomes a pass over chunk headers alone), and relabels every
 * later gate of the stage through sigma.  out (may be NULL; room for `count`)
 * receives the remaining gates as "DenseMatrix" gates without controls,
 * targets ascending, and *out_count their number; perm_dst (may be NULL;
 * n - chunk_log2 entries) gets the destination of each chunk-index bit and
 * *perm_flip the bits flipped after the moves:
 *   sigma(c) = perm_flip ^ sum_b bit(c, b) << perm_dst[b],
 *   stored amplitude i  ==  true amplitude ((sigma(i >> chunk_log2) << chunk_log2) | (i & (2^chunk_log2 - 1))).
 * The engine does this unless QOMPSIM_PERMUTE_CHUNKS=0. */
qs_status qs_stage_chunk_permutation(const qs_gate *gates, size_t count, uint32_t n, uint32_t chunk_log2,
                                     int reference_controls, qs_gate *out, size_t *out_count,
                                     int32_t *perm_dst, uint64_t *perm_flip);

/* Planner results: number of stages and blocks; one stage's gate ids,
 * block->group map (nblocks entries, may be NULL) and group count. */
qs_status qs_get_plan_info(qs_state *h, uint32_t *nstages, uint32_t *nblocks);
qs_status qs_get_stage(qs_state *h, uint32_t stage, uint32_t *gate_ids, uint32_t cap,
                       uint32_t *count, uint32_t *block_to_group, uint32_t *num_groups);

/* apply_circuit() -- compressed_state.hpp:840-937 with process_SV_group_GPU
 * (compressed_state_cuda.cu:143-381): every stage over its active groups,
 * as fused device passes over the HBM-resident store. */
qs_status qs_apply_circuit(qs_state *h);

/* get_decompressed_state_vector() -- compressed_state.hpp:1683-1707: dense
 * complex128 (interleaved re, im; 2*2^n doubles) into host memory.
 * renormalize != 0 divides by the norm as the reference does. */
qs_status qs_get_vector(qs_state *h, double *out, int renormalize);

/* Amplitudes [first, first + count) of the same dense vector (2*count
 * doubles); first and count are multiples of the chunk size 2^chunk_log2.
 * Lets a caller stream a state larger than host memory allows at once
 * (fidelity in slices); the reference reads only whole vectors.  out may be
 * host memory or device memory of the state's GPU (the copy direction is
 * taken from the pointer), so a slice can be compared on the device. */
qs_status qs_get_amplitudes(qs_state *h, uint64_t first, uint64_t count, double *out, int renormalize);

/* sampling_blockwise(sampling_count, random_seed) -- compressed_state.hpp:
 * 1600-1681, one rank: n_shots basis-state indices into out[n_shots].  The
 * per-block FP64 masses (sequential sums of x*x + y*y) and the searches
 * inside blocks run on the device; the shot split over blocks
 * (std::binomial_distribution on std::mt19937_64(seed)), the uniform draws
 * (std::mt19937_64(seed + 1)) and the final std::shuffle follow the
 * reference's order, so equal decoded amplitudes give equal samples.
 * QS_ERR_DOMAIN when the total mass is not finite and positive (the
 * reference's std::domain_error). */
qs_status qs_sample_blockwise(qs_state *h, uint32_t n_shots, uint32_t seed, uint64_t *out);

/* Squared norm of the compressed state, accumulated in FP64. */
qs_status qs_norm_squared(qs_state *h, double *out);

/* Pauli expectation sums on the compressed state, FP64 accumulation: for
 * term t with flip mask x_masks[t] (qubits carrying X or Y) and sign mask
 * z_masks[t] (qubits carrying Z or Y), out[2t] + i out[2t+1] =
 * sum_x conj(psi[x ^ x]) (-1)^{popcount(x & z)} psi[x].  The caller applies
 * i^(number of Y factors) and the coefficients, and divides by the squared
 * norm (the term with both masks 0).  Replaces Observable /
 * get_expectation_value on the reference's uncompressed states
 * (src/cppsim/observable.hpp:80); the reference has no expectation value on
 * its compressed state.  A term may flip at most tile_log2 - chunk_log2
 * qubits at or above the chunk size. */
qs_status qs_expectation_pauli(qs_state *h, const uint64_t *x_masks, const uint64_t *z_masks, size_t nterms,
                               double *out);

/* Transition sums between two compressed states of the same geometry (qubits,
 * block, chunk, dtype, error bounds): out[2t] + i out[2t+1] =
 * sum_x conj(bra[x ^ x_t]) (-1)^{popcount(x & z_t)} ket[x], FP64
 * accumulation, no normalisation.  The adjoint sweep's <lambda|P|psi> on
 * compressed states; the reference has no counterpart (its gradients run on
 * uncompressed states, src/vqcsim/parametric_circuit.cpp:180-306). */
qs_status qs_transition_pauli(const qs_state *bra, qs_state *ket, const uint64_t *x_masks,
                              const uint64_t *z_masks, size_t nterms, double *out);

/* out := (sum_t c_t Z^{z_masks[t]}) in for a diagonal observable (Z strings
 * only; coefs complex interleaved, at most 256 terms): one fused pass that
 * decodes in's store, multiplies every amplitude by h(x) = sum_t c_t
 * (-1)^{popcount(x & z_t)} and encodes into out's store (previous contents
 * of out are replaced; out keeps in's zero-block mask).  in and out are
 * distinct states of the same geometry.  This is Observable::apply_to_state
 * (src/cppsim/observable.cpp) restricted to diagonal terms, on compressed
 * states, for the adjoint sweep's lambda = H psi. */
qs_status qs_apply_diagonal_pauli_sum(qs_state *out, const qs_state *in, const uint64_t *z_masks,
                                      const double *coefs, size_t nterms);

/* out := (sum_t c_t P_t) in for general Pauli strings P_t = i^{ny} X^{x_t}
 * Z^{z_t} (coefs complex interleaved with i^{ny} folded in, so that
 * (P_t in)[x] = (-1)^{popcount(y & z_t)} in[y], y = x ^ x_t): passes that
 * decode in's store and accumulate the terms into out's (terms grouped so
 * that each group's flip qubits fit one tile).  Observable::apply_to_state
 * (src/cppsim/observable.cpp) on compressed states: the adjoint sweep's
 * lambda = H psi for observables with X / Y terms.  in and out are distinct
 * states of the same geometry in HBM; afterwards every block of out is
 * stored. */
qs_status qs_apply_pauli_sum(qs_state *out, qs_state *in, const uint64_t *x_masks, const uint64_t *z_masks,
                             const double *coefs, size_t nterms);

/* Backward sweep of the adjoint gradient over two compressed states, the
 * compressed counterpart of qs_dense_adjoint: gates (already inverted, in
 * the order to apply) act on both psi and lam; before a gate with slots[i]
 * >= 0, out[2 slots[i]], out[2 slots[i] + 1] += sum_x conj(lam[x ^ gen_x])
 * (-1)^{popcount(x & gen_z)} psi[x].  The reference's
 * ParametricQuantumCircuit::backprop_inner_product
 * (src/vqcsim/parametric_circuit.cpp:180-266) on the uncompressed state is
 * what it computes; the reference has no gradient on its compressed state.
 * Each fused pass decodes tiles of both stores, applies its gates and sums,
 * and re-encodes both.  psi and lam are distinct states of one geometry in
 * HBM on one stream; out (2 * nslots doubles) is overwritten. */
qs_status qs_adjoint(qs_state *psi, qs_state *lam, const qs_gate *gates, const int32_t *slots, const uint64_t *gen_x,
                     const uint64_t *gen_z, size_t count, double *out, uint32_t nslots);

/* One dense k-qubit gate (k = 4 or 5: the gates optimize(c, block_size=k)
 * fuses; matrix bit i <-> targets[i], row-major 2^k x 2^k complex128,
 * interleaved) applied to the compressed state at once, as a stage of its
 * own: groups of blocks differing in the gate's qubits >= block_size, the
 * reference's zero-mask rule at the end.  One fused pass over tiles of 2^12
 * amplitudes (at most 12 - chunk_log2 of the targets above the chunk):
 * complex64 multiplies each tile by the gate on the tensor cores (tcgen05
 * tf32 MMAs with a 3xTF32 split, FP32 accumulation), complex128 on the CUDA
 * cores.  The reference's compressed engine rejects gates on more than two
 * qubits (compressed_state.hpp:1003-1007); this is an extension.  The
 * statistics describe this pass (qs_get_stats). */
qs_status qs_apply_dense_gate(qs_state *h, const uint32_t *targets, uint32_t k, const double *matrix);

/* Zero-block mask: out[b] = 1 when block b is stored (the reference's
 * block_pointers[b] != nullptr, compressed_state.hpp:18-19, 319-325). */
qs_status qs_get_zero_mask(qs_state *h, uint8_t *out);

/* blocks_bytes (compressed_state.hpp:19): stored bytes per block (0 for a
 * zero block): chunk payloads plus their 16-byte chunk headers. */
qs_status qs_get_block_bytes(qs_state *h, uint64_t *out);

/* get_max_SV_bytes() -- compressed_state.hpp:439-445: the largest total
 * over the initial state and every stage end. */
qs_status qs_get_max_sv_bytes(qs_state *h, uint64_t *out);

/* Totals after the initial state and after each stage ("Total SV bytes",
 * compressed_state.hpp:374-437).  *count receives the number available. */
qs_status qs_get_sv_bytes_history(qs_state *h, uint64_t *out, size_t cap, size_t *count);

/* get_total_times() -- python/cppsim_wrapper.cpp:503-515, the same ten keys
 * in this order: decomp, gate, comp, fused_swap, allgather, hmalloc, dmalloc,
 * h2d, d2h, dfree (seconds).  "gate" holds the fused passes' device time,
 * which also contains decoding and encoding; decomp/comp stay 0. */
qs_status qs_get_total_times(qs_state *h, double out[10]);

qs_status qs_get_stats(qs_state *h, qs_stats *out);

/* Serialise the compressed store (zero mask, chunk headers and payloads) into
 * host memory and back.  With buf == NULL, qs_export_store only reports the
 * size.  These replace the host-resident block_pointers of the reference. */
qs_status qs_export_store(qs_state *h, void *buf, uint64_t cap, uint64_t *size);
qs_status qs_import_store(qs_state *h, const void *buf, uint64_t size);

/* Multi-rank exchange (replaces apply_fused_swap's compressed block
 * send/recv, compressed_state.hpp:1396-1546, for one swapped qubit pair):
 * a rank holding global qubit bit b swaps it with its local qubit `qubit`
 * (chunk bits <= qubit < n) by sending the half of its store whose
 * amplitude-index bit `qubit` equals 1-b and receiving the partner's half
 * into the same positions.  qs_export_half packs the half whose bit equals
 * `value` (chunk headers and compressed payloads, no decoding) into a
 * 128-byte aligned DEVICE buffer; with dev_buf == NULL it only reports the
 * size.  qs_import_half writes a packed half received from a partner of the
 * same geometry and codec into the positions whose bit equals `value`
 * (payloads appended to the current arena, headers rewritten, blocks marked
 * stored, per-block bytes recomputed); QS_ERR_CORRUPT when the buffer does
 * not match or a header points outside it.  Both synchronise the stream.
 * qs_set_zero_vector makes the state the zero vector (every block unstored):
 * the initial store of ranks that do not hold |0...0>. */
qs_status qs_export_half(qs_state *h, uint32_t qubit, uint32_t value, void *dev_buf, uint64_t cap, uint64_t *size);
qs_status qs_import_half(qs_state *h, uint32_t qubit, uint32_t value, const void *dev_buf, uint64_t size);
qs_status qs_set_zero_vector(qs_state *h);

/* Failure-path self-test of the bounded device waits (the staged and dense
 * tensor-core passes wait on mbarriers with an iteration limit, after which
 * the pass sets its error flag and the call returns QS_ERR_TIMEOUT): one CTA
 * arms an mbarrier that nothing completes and waits at most `tries` times.
 * *gave_up = 1 when the wait gave up, as it must; the context stays usable. */
qs_status qs_selftest_bounded_wait(uint32_t tries, int32_t *gave_up);

/* Device-side checkpoints of the compressed store (zero mask, per-block
 * bytes, chunk headers and the payload in use): qs_checkpoint copies the
 * current store into slot (0..63, allocated on first use, regrown when the
 * store has grown), qs_restore copies it back.  The reference has no
 * checkpoint of its compressed state; these are the stage checkpoints of
 * the adjoint and a cheap way to rerun a circuit from a saved state. */
qs_status qs_checkpoint(qs_state *h, uint32_t slot);
qs_status qs_restore(qs_state *h, uint32_t slot);
qs_status qs_free_checkpoint(qs_state *h, uint32_t slot);

/* Reset to |basis> (basis < 2^n); the reference only has |0...0>. */
qs_status qs_set_basis_state(qs_state *h, uint64_t basis);

/* Load a dense complex128 vector (2*2^n doubles, host) into the compressed
 * store, compressing it.  A block is stored when any amplitude is non-zero. */
qs_status qs_load_vector(qs_state *h, const double *vec);

/* ------------------------------------------------- uncompressed (dense) */

/* QuantumState(qubit_count) on the device, initialised to |0...0>. */
qs_status qs_dense_create(qs_dense **out, uint32_t n, qs_dtype dtype);
qs_status qs_dense_destroy(qs_dense *h);
qs_status qs_dense_set_stream(qs_dense *h, void *cuda_stream);

/* QuantumCircuit::update_quantum_state(state) (src/cppsim/circuit.cpp:23-34):
 * the gates are applied in order, grouped into fused tile passes. */
qs_status qs_dense_apply_gates(qs_dense *h, const qs_gate *gates, size_t count);

/* The plain path: one full-vector kernel per gate, as the reference's
 * gpusim kernels do (e.g. double_qubit_dense_matrix_gate_host,
 * src/gpusim/update_ops_multi.cu:373).  Used as the per-gate baseline. */
qs_status qs_dense_apply_gates_pergate(qs_dense *h, const qs_gate *gates, size_t count);

/* QuantumState::get_vector / load (state.hpp:445-1045); 2*2^n doubles. */
qs_status qs_dense_get_vector(qs_dense *h, double *out);
/* Amplitudes [first, first + count) as complex128 (2*count doubles); out
 * may be host memory or device memory of the state's GPU. */
qs_status qs_dense_get_amplitudes(qs_dense *h, uint64_t first, uint64_t count, double *out);
qs_status qs_dense_set_vector(qs_dense *h, const double *in);
qs_status qs_dense_set_basis_state(qs_dense *h, uint64_t basis);
qs_status qs_dense_norm_squared(qs_dense *h, double *out);

/* The same Pauli expectation sums on the uncompressed state. */
qs_status qs_dense_expectation_pauli(qs_dense *h, const uint64_t *x_masks, const uint64_t *z_masks, size_t nterms,
                                     double *out);

/* dst := src (same size and dtype). */
qs_status qs_dense_copy(qs_dense *dst, const qs_dense *src);

/* out := sum_t c_t P_t in, P_t the Pauli string with flip mask x_masks[t] and
 * sign mask z_masks[t] acting as P|y> = (-1)^{|y & z|} |y ^ x|; coefs holds
 * the complex c_t (interleaved re, im), with any i^(number of Y) folded in.
 * Observable::apply_to_state of the reference (used by its backprop,
 * src/vqcsim/parametric_circuit.cpp:268-306). */
qs_status qs_dense_apply_pauli_sum(qs_dense *out, const qs_dense *in, const uint64_t *x_masks,
                                   const uint64_t *z_masks, const double *coefs, size_t nterms);

/* Transition sums out[2t] + i out[2t+1] = sum_x conj(bra[x ^ x_t]) (-1)^{|x & z_t|} ket[x]. */
qs_status qs_dense_transition_pauli(const qs_dense *bra, qs_dense *ket, const uint64_t *x_masks,
                                    const uint64_t *z_masks, size_t nterms, double *out);

/* Adjoint backward sweep over two states (reverse-mode differentiation of a
 * parametric circuit; the reference's backprop_inner_product,
 * src/vqcsim/parametric_circuit.cpp:180-266, restated as fused tile passes).
 * gates[0..count) are applied in order to both psi and lam -- the caller
 * lists the inverse gates U_k^dagger in reverse circuit order.  Before gate
 * i with slots[i] >= 0, the sums sum_x conj(lam[x ^ gen_x[i]])
 * (-1)^{|x & gen_z[i]|} psi[x] are added to out[2 slot] + i out[2 slot + 1]
 * (nslots slots, zeroed by the call).  For a rotation exp(i theta/2 P) the
 * derivative of <psi|H|psi> is then -Im(i^(number of Y in P) * sum). */
qs_status qs_dense_adjoint(qs_dense *psi, qs_dense *lam, const qs_gate *gates, const int32_t *slots,
                           const uint64_t *gen_x, const uint64_t *gen_z, size_t count, double *out,
                           uint32_t nslots);

/* Device pointer of the amplitudes (interleaved re, im of the dtype). */
qs_status qs_dense_device_ptr(qs_dense *h, void **out);

/* ------------------------------------------------------------- codec */

/* Quantiser parameters (m, L) the engine derives from eps_rel / eps_abs. */
qs_status qs_codec_params(qs_dtype dtype, double eps_rel, double eps_abs,
                          int32_t *m, int32_t *L);

/* Encode nchunks chunks of 2^chunk_log2 amplitudes (vals: interleaved re, im
 * of the dtype, host memory) on the device and decode them again.  words
 * receives each chunk's payload at a stride of 2^(chunk_log2+1) words, bases
 * and widths its frame of reference, decoded the round-tripped values.  It
 * exists to check the device codec against its CPU statement bit for bit;
 * the reference has no counterpart (Bitcomp is a closed library). */
qs_status qs_codec_test(qs_dtype dtype, double eps_rel, double eps_abs, uint32_t chunk_log2,
                        const void *vals, uint64_t nchunks, uint32_t *words, int32_t *bases,
                        uint32_t *widths, void *decoded);

/* Allocation-free variant of qs_codec_test, for callers that cannot call
 * cudaMalloc: code that runs inside another framework's memory pool, that
 * has reserved all device memory up front, or that must not allocate (an
 * allocation may synchronise the device) in the middle of a running
 * pipeline.  No counterpart in the reference.
 *
 * All pointers are DEVICE pointers owned by the caller: d_vals holds
 * nchunks * 2^(chunk_log2+1) values of the dtype (interleaved re, im);
 * d_bases / d_widths receive each chunk's frame of reference and d_decoded the
 * round-tripped values, exactly as qs_codec_test returns them.  The packed
 * words between encode and decode live in a file-scope device array of
 * 4 MiB that every GPU loading the library holds until the process exits;
 * a call may cover at most 2^20 / 2^(chunk_log2+1) chunks (larger calls
 * return QS_ERR_ARG, nothing is launched).  The call allocates nothing,
 * enqueues one kernel on `stream` (a cudaStream_t, NULL = default stream)
 * and does not synchronise.  Its first call on a device looks up the
 * array's device address with that device current, so make that first call
 * before any stream capture.  Every later call made outside a capture looks
 * the address up again (after cudaDeviceReset, or under another context on
 * the same device, the array has a new address); a call inside a capture
 * uses the address that the last call outside one found.  Every call shares the
 * one array: calls that overlap on the GPU (different streams, no ordering
 * between them) race on it.  Nothing in the array needs to start at zero;
 * it keeps the last call's words.  Errors are reported through
 * qs_dense_last_error(NULL). */
qs_status qs_codec_roundtrip_noalloc(qs_dtype dtype, double eps_rel, double eps_abs, uint32_t chunk_log2,
                                     const void *d_vals, uint64_t nchunks, int32_t *d_bases,
                                     uint32_t *d_widths, void *d_decoded, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QOMPSIM_H */
