// Internal interface between the host engine (engine.cpp) and the device code
// (kernels.cu).  Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace qs {

// Largest chunk: 2^8 amplitudes = 512 real components = 16 per lane.
constexpr int kMaxChunkLog2 = 8;
constexpr int kMinChunkLog2 = 4;
constexpr int kMaxPerLane = (2 << kMaxChunkLog2) / 32;
// Largest tile: 2^14 amplitudes; at most kMaxTileQubits qubits above the chunk.
constexpr int kMaxTileLog2 = 14;
constexpr int kMaxTileQubits = 10;
constexpr int kPassThreads = 256;

// Header of one encoded chunk (16 bytes).  offset is a byte offset into the
// payload arena; the payload is 128 * rows bytes (see codec.cuh).
struct ChunkMeta {
    uint64_t offset;
    int32_t base;
    uint32_t width;
};
static_assert(sizeof(ChunkMeta) == 16, "chunk header is 16 bytes");

// A gate as the device applies it: nq (1 or 2) qubits in ascending order,
// matrix index bit i <-> q[i], complex128 row-major interleaved.  tpos[i] is
// the qubit's bit position inside the tile, or -1 when the qubit is outside
// the tile (then the gate is diagonal in that qubit and the tile's fixed bit
// selects the sub-matrix).  diag != 0: the matrix is diagonal.
struct KGate {
    int32_t nq;
    int32_t q[2];
    int32_t tpos[2];
    int32_t diag;
    int32_t mixmask;    // bit i: the gate mixes amplitudes along q[i]
    int32_t pad;
    double m[32];
};

// Register blocking: a sweep applies gates g0..g1-1 of a pass in one pass
// over the tile in shared memory.  Each thread holds 2^RB amplitudes whose
// tile indices differ in the sweep's RB tile bits `sbits` (ascending); every
// gate of the sweep mixes amplitudes only along those bits (diagonal action
// on any other bit is allowed).  RB = 3 for complex128, 4 for complex64.
constexpr int kRegBitsF64 = 3;
constexpr int kRegBitsF32 = 4;
constexpr int kMaxRegBits = 5;
struct Sweep {
    int32_t g0, g1;
    int32_t sbits[6];
};
// Threads of the fused pass kernels (compressed and dense): 4 warps, three
// CTAs per SM, so that a thread can hold 2^RB amplitudes in registers.
constexpr int kSweepThreads = 128;

// A gate resolved against its sweep (host-built).  Register bits k0/k1 index
// the sweep bits; the gate's other qubits are fixed for a register group and
// select one of 2^nsel pre-computed sub-matrix variants: selector source
// sel[j] < 64 is a tile bit (its value comes from the group), sel[j] >= 64 is
// qubit sel[j]-64 outside the tile (its value comes from the tile).
enum : uint8_t { OP_SCALAR = 0, OP_D2 = 1, OP_M2 = 2, OP_D4 = 3, OP_M4 = 4 };
constexpr int kMaxSel = 4;
struct ROp {
    uint8_t kind;
    uint8_t k0, k1;      // register bits; for D4/M4 k0 <-> matrix bit 0
    uint8_t nsel;        // 0..kMaxSel selector bits
    uint8_t sel[kMaxSel];
    uint32_t mat;        // pool index of variant 0 (complex entries)
    uint32_t vstride;    // complex entries per variant: 1, 2, 4 or 16
};
static_assert(sizeof(ROp) == 16, "ROp is one 16-byte load");
static_assert(sizeof(KGate) == 288, "KGate layout");

struct CodecParams {
    int32_t m;      // mantissa bits kept (relative step 2^-m)
    int32_t L;      // absolute step 2^-L in the linear region
};

// A permutation of chunk indices (the amplitude-index bits >= C) made of bit
// moves and bit flips: SWAP and X gates on qubits >= C move whole chunks, so
// they are applied by rewriting chunk headers, never by decoding payloads.
//   perm(c) = ((c & keep) | sum_k bit(c, src[k]) << dst[k]) ^ flip
constexpr int kMaxPermBits = 40;
struct ChunkPerm {
    uint64_t keep;          // bits that stay in place (all ones: identity)
    uint64_t flip;          // bits flipped after the moves
    int32_t nmove;
    int8_t src[kMaxPermBits], dst[kMaxPermBits];
};

// One fused pass over the compressed store.
struct PassArgs {
    int32_t n, B, C, j;                 // qubits, block log2, chunk log2, tile qubits above C
    int32_t tq[kMaxTileQubits];         // tile qubits minus C (chunk-index bit), ascending
    uint64_t n_tiles;                   // 2^(n - C - j)
    const ROp *ops;
    const void *pool;                   // double2 (complex128) or float2 (complex64)
    const Sweep *sweeps;
    int32_t nsweeps;
    int32_t rb;                         // register bits of the sweeps (3 or the dtype's RB)
    CodecParams codec;
    const ChunkMeta *meta_in;
    const uint32_t *arena_in;
    ChunkMeta *meta_out;
    uint32_t *arena_out;
    unsigned long long *bump;           // bytes used in arena_out
    uint64_t capacity;                  // bytes of arena_out
    const uint32_t *block_to_group;     // stage's map
    const uint8_t *group_active;
    const uint8_t *mask;                // zero-block mask at stage start
    int32_t first_pass, final_pass, exact_zero;
    uint32_t *block_nz;                 // final pass: any non-zero in block
    unsigned long long *block_bytes;    // final pass: stored bytes of block
    int32_t *error;                     // 1 = arena overflow
    unsigned long long *stats;          // [0] bytes read [1] bytes written [2] tiles
    ChunkPerm perm;                     // chunk c of the pass is stored as chunk perm(c)
};

// A pass that only permutes chunk headers: meta_out[perm(c)] = meta_in[c]
// for the chunks of active groups (the payload arena is shared).
struct PermPassArgs {
    int32_t B, C;
    uint64_t nchunks;
    const ChunkMeta *meta_in;
    ChunkMeta *meta_out;
    const uint32_t *block_to_group;
    const uint8_t *group_active;
    const uint8_t *mask;
    int32_t first_pass, final_pass;
    uint32_t *block_nz;
    unsigned long long *block_bytes;
    unsigned long long *stats;
    ChunkPerm perm;
};

// One fused pass over a dense state vector (in place).
struct DensePassArgs {
    int32_t n, C, j;
    int32_t tq[kMaxTileQubits];
    uint64_t n_tiles;
    const ROp *ops;
    const void *pool;
    const Sweep *sweeps;
    int32_t nsweeps;
    int32_t rb;
    void *state;
};

// A Pauli string as the expectation kernels read it: P|x> = i^ny (-1)^{|x & z|} |x ^ x_flip>.
// Tile-local masks (bits of the tile index) plus the parity of z-qubits that
// lie outside the tile (taken from the tile's base amplitude).
struct PauliTerm {
    uint32_t xt, zt;   // flip / sign masks over tile bits
    uint64_t zo;       // sign mask over qubits outside the tile (global bit positions)
    uint64_t xg, zg;   // the same string over global qubits (dense kernel)
};

// One read-only pass over the compressed store accumulating, for each term t,
// S_t = sum_x conj(psi_{x ^ xflip}) (-1)^{|x & z|} psi_x into out[2t], out[2t+1].
struct ExpectArgs {
    int32_t n, B, C, j;
    int32_t tq[kMaxTileQubits];
    uint64_t n_tiles;
    const ChunkMeta *meta;
    const uint32_t *arena;
    const uint8_t *mask;
    CodecParams codec;
    const PauliTerm *terms;
    int32_t nterms;
    double *out;
};

// Backward (adjoint) pass over two uncompressed states psi and lam: gates are
// applied in the listed order (the caller lists U_k^dagger in reverse circuit
// order); before a gate with slot >= 0, S_slot = sum_x conj(lam[x ^ gen.x])
// (-1)^{|x & gen.z|} psi[x] is accumulated into out[2 slot], out[2 slot + 1].
struct AdjGate {
    KGate g;           // the gate to apply (tile positions resolved)
    PauliTerm gen;     // generator of the parametric gate (tile-local masks)
    int32_t slot;      // -1: no derivative at this gate
    int32_t pad;
};
struct AdjPassArgs {
    int32_t n, C, j;
    int32_t tq[kMaxTileQubits];
    uint64_t n_tiles;
    const AdjGate *gates;
    int32_t ngates;
    void *psi;
    void *lam;
    double *out;
    int32_t nslots;
};

// ---- launchers (kernels.cu); all asynchronous on `stream` ----
cudaError_t launch_adjoint_pass(bool f64, const AdjPassArgs &a, cudaStream_t stream);
cudaError_t launch_dense_transition(bool f64, const void *bra, const void *ket, int n, const PauliTerm *terms,
                                    int nterms, double *out, cudaStream_t stream);
// out = sum_t coef_t P_t in (coefs complex interleaved; PauliTerm global masks, ny folded into coefs)
cudaError_t launch_dense_pauli_sum(bool f64, const void *in, void *out, int n, const PauliTerm *terms,
                                   const double *coefs, int nterms, cudaStream_t stream);
cudaError_t launch_expect(bool f64, const ExpectArgs &a, cudaStream_t stream);
cudaError_t launch_dense_expect(bool f64, const void *state, int n, const PauliTerm *terms, int nterms, double *out,
                                cudaStream_t stream);
cudaError_t launch_pass(bool f64, const PassArgs &a, int tile_log2, cudaStream_t stream);
cudaError_t launch_perm_pass(const PermPassArgs &a, cudaStream_t stream);
cudaError_t launch_dense_pass(bool f64, const DensePassArgs &a, int tile_log2, cudaStream_t stream);
cudaError_t launch_pergate(bool f64, void *state, int n, const KGate *gate_dev, cudaStream_t stream);

cudaError_t launch_stage_begin(const uint32_t *block_to_group, const uint8_t *mask, uint32_t nb,
                               uint8_t *group_active, uint32_t num_groups, uint32_t *block_nz,
                               unsigned long long *block_bytes, unsigned long long *active_blocks,
                               cudaStream_t stream);
cudaError_t launch_stage_end(const uint32_t *block_to_group, const uint8_t *group_active, uint32_t nb,
                             const uint32_t *block_nz, const unsigned long long *block_bytes_acc,
                             uint8_t *mask, unsigned long long *block_bytes,
                             unsigned long long *history_slot, cudaStream_t stream);

// Decode chunks [chunk0, chunk0 + nchunks) into complex128 (interleaved).
cudaError_t launch_readout(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask,
                           int B, int C, CodecParams codec, uint64_t chunk0, uint64_t nchunks,
                           double *out, double scale, cudaStream_t stream);
// sum |a|^2 over the stored blocks (FP64 accumulation); *out must be zeroed.
cudaError_t launch_norm(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask,
                        int B, int C, CodecParams codec, uint64_t nchunks, double *out,
                        cudaStream_t stream);
// Encode complex128 chunks (host layout interleaved, on device) into the
// store: chunks [chunk0, chunk0 + nchunks) read from `vals`.
cudaError_t launch_encode(bool f64, const double *vals, int B, int C, CodecParams codec,
                          uint64_t chunk0, uint64_t nchunks, ChunkMeta *meta, uint32_t *arena,
                          unsigned long long *bump, uint64_t capacity, uint32_t *block_nz,
                          unsigned long long *block_bytes, int32_t *error, cudaStream_t stream);
cudaError_t launch_dense_norm(bool f64, const void *state, uint64_t dim, double *out, cudaStream_t stream);
cudaError_t launch_dense_to_c128(bool f64, const void *state, uint64_t dim, double *out, cudaStream_t stream);
cudaError_t launch_c128_to_dense(bool f64, const double *in, uint64_t dim, void *state, cudaStream_t stream);
cudaError_t launch_sum_mask_bytes(const uint8_t *mask, const unsigned long long *block_bytes, uint32_t nb,
                                  unsigned long long *out, cudaStream_t stream);

// Device codec round trip of whole chunks (tests of CPU/GPU bit identity).
cudaError_t launch_codec_test(bool f64, const void *vals, int C, CodecParams codec, uint64_t nchunks,
                              uint32_t *words, int32_t *bases, uint32_t *widths, void *decoded,
                              cudaStream_t stream);

// Allocation-free variant of launch_codec_test: the packed words live in a
// file-scope device array of noalloc_scratch_words() words.
cudaError_t launch_codec_roundtrip_noalloc(bool f64, const void *vals, int C, CodecParams codec, uint64_t nchunks,
                                           int32_t *bases, uint32_t *widths, void *decoded, cudaStream_t stream);
uint64_t noalloc_scratch_words();

int sm_count();

}  // namespace qs
