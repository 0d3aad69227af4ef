// Internal interface between the host engine (engine.cpp) and the device code
// (kernels.cu).  Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace qs {

// Largest chunk: 2^8 amplitudes = 512 real components = 16 per lane.
constexpr int kMaxChunkLog2 = 8;
// Arena space a pass-kernel CTA takes at once (when the arena holds at least
// eight per CTA), sub-allocated to its tiles without the shared counter.
constexpr uint64_t kArenaSlabBytes = 256 << 10;
constexpr int kMinChunkLog2 = 4;
constexpr int kMaxPerLane = (2 << kMaxChunkLog2) / 32;
// Largest tile: 2^14 amplitudes; at most kMaxTileQubits qubits above the chunk.
constexpr int kMaxTileLog2 = 14;
constexpr int kMaxTileQubits = 10;
// Threads of the per-chunk codec kernels (readout, norm, encode, codec tests):
// one warp per chunk, four warps per CTA.
constexpr int kPassThreads = 128;

// Header of one encoded chunk (16 bytes).  offset is a byte offset into the
// payload arena; the payload is 128 * rows bytes (see codec.cuh).
// Invariant every device reader relies on: the header of a chunk is read only
// when its block is stored (zero mask set) or the pass is not the first of
// its stage (every block of an active group has been written by then); the
// headers of unstored blocks are zero (offset 0, width 0) after an import.
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

// Register blocking: a sweep applies ops g0..g1-1 of a pass in one pass
// over the tile in shared memory.  Each thread holds 2^RB amplitudes whose
// tile indices differ in the sweep's RB tile bits `sbits` (ascending); every
// op of the sweep mixes amplitudes only along those bits (diagonal action on
// any other bit is allowed).  RB = 4 for both precisions: 16 amplitudes per
// group keep every op's arithmetic independent across the group, which is
// what hides the latency of the op stream.
constexpr int kRegBits = 4;
constexpr int kRegBitsF64 = kRegBits;
constexpr int kRegBitsF32 = kRegBits;
constexpr int kMaxRegBits = kRegBits;
struct Sweep {
    int32_t g0, g1;
    int32_t sbits[6];
};
// Threads of the fused pass kernels (compressed and dense): 4 warps per CTA.
constexpr int kSweepThreads = 128;

// One register op (host-built, 16 bytes).  `code` names the action and the
// register bits it acts on; the gate's other qubits are fixed for a register
// group and select one of 2^nsel (nsel <= 8) pre-computed variants: sel[j] is a bit
// position in the group word W = (tile index of the group's element 0) |
// (outer selector bits << tile bits), unused slots hold 31 (always 0 in W).
//   OPC_SCALAR           z *= m[0]                (lazy: one factor per group)
//   OPC_D2  + k          diag(m0, m1) on bit k
//   OPC_D2H + k          diag(1,  m0) on bit k    (only the bit-1 half)
//   OPC_M2  + k          2x2 matrix m0..m3 on bit k
//   OPC_X   + k          swap the halves of bit k (Pauli X, no arithmetic)
//   OPC_D4  + (a*8+b)    diag(m0..m3) on bits a < b (matrix bit 0 <-> a)
//   OPC_D4H + (a*8+b)    diag(1, m0, m1, m2) on bits a < b
//   OPC_M4  + (a*8+b)    4x4 matrix m0..m15 on bits a < b
//   OPC_SWAP + (a*8+b)   exchange bits a and b (no arithmetic)
//   OPC_ACC              zh *= m[0]               (a pending bit-1 factor)
//   OPC_D2HP + k         diag(1, zh m0) on bit k, then zh = 1: the last of a
//                        run of half-diagonals on one bit inside a sweep, the
//                        others of which became OPC_ACC (fuse_half_chains)
//   OPC_SUM              two-store sweeps only: derivative sum, see below
enum : uint8_t {
    OPC_SCALAR = 0, OPC_D2 = 8, OPC_D2H = 16, OPC_M2 = 24, OPC_X = 32, OPC_ACC = 40, OPC_D2HP = 48,
    OPC_D4 = 64, OPC_D4H = 96, OPC_M4 = 128, OPC_SWAP = 160, OPC_SUM = 224
};
// OPC_SUM in a two-store sweep (groups v of store A and w of store B at the
// same tile positions): sums[slot] += f * sum_s conj(w[s ^ xs]) (-1)^{|s & zs|} v[s],
// xs / zs = the generator's flip / Z qubits among the register bits
// (ROp.pad = xs << 4 | zs), slot = ROp.vstride, and f = +-1 (variant real
// part) the sign of its Z qubits among the selector bits.  The stores' lazy
// scalar factors enter as conj(zB) zA.
constexpr int kMaxSel = 8;
constexpr uint8_t kSelNone = 31;
// sel[0] with this bit set: the selectors are given as at most two runs of
// consecutive W bits (sel[0] & 31 = start of the first, sel[1] its length,
// sel[2] / sel[3] the second), variant bit j = the j-th selector in order.
constexpr uint8_t kSelRuns = 0x80;
struct ROp {
    uint8_t code;
    uint8_t nsel;        // 0..kMaxSel selector bits
    uint8_t vstride;     // complex entries per variant (0..16)
    uint8_t pad;
    uint8_t sel[kMaxSel];
    uint32_t mat;        // pool index of variant 0 (complex entries)
};
// Outer qubits (outside the tile) that select variants: at most this many per
// pass, so that tile bits + outer bits stay below bit 31 of W.
constexpr int kMaxOuterSel = 16;
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

// Diagonal Pauli sum applied inside a tile pass: each element x of a tile is
// multiplied by h(x) = sum_t c_t (-1)^{|x & z_t|}; zt is the tile-local mask
// and zo the mask of qubits outside the tile (PauliTerm fields).
constexpr int kMaxDiagTerms = 256;
struct PauliTerm;
struct DiagSum {
    const PauliTerm *terms;   // xt = xg = 0
    const double *coefs;      // complex, interleaved
    int32_t nterms;
};

// A dense k-qubit gate applied over a whole tile of 2^kDenseTileLog2
// amplitudes (kMinDenseK <= k <= kMaxDenseK): the tile's 2^(12-k) columns
// (patterns of its other bits) are the rows of one GEMM y = G x.
//   complex64:  tensor cores (tcgen05.mma kind::tf32 with a 3xTF32 split):
//               the gate as the real 2^(k+1) x 2^(k+1) matrix
//               [[Gr, -Gi], [Gi, Gr]] (row = output: Re y_0.. then Im y_0..;
//               column = input: Re x_0.. then Im x_0..), split into tf32 hi
//               and lo parts, each in the K-major unswizzled operand layout
//               of dense_k_operand_offset
//   complex128: CUDA cores, the 2^k x 2^k matrix row-major (double2)
constexpr int kMinDenseK = 4;
constexpr int kMaxDenseK = 5;
constexpr int kDenseTileLog2 = 12;
struct DenseKGate {
    int32_t k;
    int32_t pos[kMaxDenseK];    // tile bit position of matrix bit i
    const float *bhi, *blo;     // complex64 operands (2^(2k+2) floats each)
    const double *mat;          // complex128 matrix (2^(2k) complex, interleaved)
};

// Byte offset of element (row, col) of a K-major, unswizzled tcgen05
// operand with kcols columns: 8-row x 16-byte core matrices, consecutive
// along K (leading byte offset 128), 8-row groups kcols * 32 bytes apart
// (stride byte offset).
__host__ __device__ inline uint32_t dense_k_operand_offset(uint32_t row, uint32_t col, uint32_t kcols) {
    return (row >> 3) * (kcols * 32u) + (col >> 2) * 128u + (row & 7u) * 16u + (col & 3u) * 4u;
}

// One fused pass over the compressed store.
struct PassArgs {
    int32_t n, B, C, j;                 // qubits, block log2, chunk log2, tile qubits above C
    int32_t tq[kMaxTileQubits];         // tile qubits minus C (chunk-index bit), ascending
    uint64_t n_tiles;                   // 2^(n - C - j)
    const ROp *ops;
    const void *pool;                   // double2 (complex128) or float2 (complex64)
    const Sweep *sweeps;
    int32_t nsweeps;
    int32_t rb;                         // register bits of the sweeps (kRegBits)
    CodecParams codec;
    const ChunkMeta *meta_in;
    const uint32_t *arena_in;
    ChunkMeta *meta_out;
    uint32_t *arena_out;
    unsigned long long *bump;           // bytes used in arena_out
    uint64_t capacity;                  // bytes of arena_out
    uint64_t slab;                      // > 0: CTAs take arena space in slabs of this many bytes
    const uint32_t *block_to_group;     // stage's map
    const uint8_t *group_active;
    const uint8_t *mask;                // zero-block mask at stage start
    int32_t first_pass, final_pass, exact_zero;
    int32_t code_moves;                 // 1: every op is an X / SWAP register move (no arithmetic),
                                        // so the tile carries quantised codes, not values
    int32_t header_batch;               // complex64: chunk headers a warp loads at once (4 or 8)
    uint32_t *block_nz;                 // final pass: any non-zero in block
    unsigned long long *block_bytes;    // final pass: stored bytes of block
    int32_t *error;                     // 1 = arena overflow, 2 = a bounded wait for staged payloads gave up
    unsigned long long *stats;          // [0] bytes read [1] bytes written [2] tiles
    ChunkPerm perm;                     // chunk c of the pass is stored as chunk perm(c)
    int32_t nouter;                     // outer selector qubits of the pass
    int8_t outer_q[kMaxOuterSel];       // their global qubit indices (bit nb + i of W)
    DiagSum diag;                       // nterms > 0: multiply by a diagonal Pauli sum after the sweeps
    int32_t staged;                     // 1: staged_pass_kernel (payloads prefetched with bulk copies),
                                        // 0: pass_kernel (payloads copied chunk by chunk; the host-store arenas)
    DenseKGate dense;                   // k > 0: the pass applies this one gate instead of sweeps
                                        // (staged kernel, 2^kDenseTileLog2-amplitude tiles)
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
    int32_t nouter;
    int8_t outer_q[kMaxOuterSel];
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
    // optional bra store of the same geometry: S_t = sum_x conj(bra_{x ^ xflip})
    // (-1)^{|x & z|} ket_x (transition amplitudes); NULL meta_bra: bra = ket
    const ChunkMeta *meta_bra;
    const uint32_t *arena_bra;
    const uint8_t *mask_bra;
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
    // register sweeps over both tiles (nsweeps > 0: used instead of gates),
    // as in DualPassArgs
    const struct Sweep *sweeps;
    int32_t nsweeps;
    int32_t rb;
    const struct ROp *rops;
    const void *pool;
    int8_t outer_q[kMaxOuterSel];
    int32_t nouter;
};

// A pass over two compressed stores A and B of one geometry (the compressed
// adjoint: A = psi, B = lambda).  Per tile both are decoded, the ops run in
// order, and the stores are re-encoded into their output arenas.
enum : int32_t {
    DOP_GATE_A = 0,     // apply g to A
    DOP_GATE_B = 1,     // apply g to B
    DOP_GATE_AB = 2,    // apply g to both
    DOP_SUM = 3,        // sums[slot] += sum_x conj(B[x ^ xt]) (-1)^{|x & z|} A[x]
    DOP_ACCUM = 4       // B[x] += coef (-1)^{|y & z|} A[y], y = x ^ xt
};
struct DualOp {
    KGate g;
    PauliTerm term;     // xt, zt tile-local, zo outer
    double coef[2];
    int32_t kind;
    int32_t slot;
};
constexpr int kMaxDualSlots = 128;
// Register bits of the two-store sweeps: two groups (one per store) of
// 2^rb amplitudes are held at once.
constexpr int kDualRegBitsF32 = 4;
constexpr int kDualRegBitsF64 = 3;
struct DualStore {
    const ChunkMeta *meta_in;   // NULL: the store starts the pass at zero (B only)
    const uint32_t *arena_in;
    const uint8_t *mask_in;     // blocks stored at the start of the pass
    ChunkMeta *meta_out;        // NULL: not written (A only, when no op changes it)
    uint32_t *arena_out;
    unsigned long long *bump;
    uint64_t capacity;
    unsigned long long *block_bytes;  // per block: stored bytes written (accumulated)
};
struct DualPassArgs {
    int32_t n, B, C, j;
    int32_t tq[kMaxTileQubits];
    uint64_t n_tiles;
    const DualOp *ops;
    int32_t nops;
    // register sweeps over both stores (nsweeps > 0: used instead of ops):
    // gates as ROps applied to both groups, derivative sums as OPC_SUM
    const Sweep *sweeps;
    int32_t nsweeps;
    int32_t rb;                 // register bits: kDualRegBitsF32 / kDualRegBitsF64
    const ROp *rops;
    const void *pool;           // variants, complex of the store's precision
    int8_t outer_q[kMaxOuterSel];
    int32_t nouter;
    CodecParams codec;
    DualStore a, b;
    double *sums;               // 2 doubles per slot
    int32_t nslots;
    int32_t *error;             // 1 = an output arena overflowed
};

// ---- launchers (kernels.cu); all asynchronous on `stream` ----
cudaError_t launch_dual_pass(bool f64, const DualPassArgs &a, cudaStream_t stream);
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
// Shared memory of one staged_pass_kernel CTA for tiles of 2^(C+j) amplitudes.
size_t staged_pass_smem_bytes(bool f64, int C, int j, uint32_t nblocks);
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
// Sequential FP64 |a|^2 sum of every block (block_mass[nblocks]) and the
// running sum at the start of every chunk (prefix[nchunks]); 0 for zero blocks.
cudaError_t launch_block_mass(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B,
                              int C, CodecParams codec, uint32_t nblocks, double *prefix, double *block_mass,
                              cudaStream_t stream);
// For each shot s: the first amplitude of block shot_block[s] whose cumulative
// |a|^2 reaches rin[s] (clamped to the block); out[s] = its global index.
cudaError_t launch_sample_in_block(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask,
                                   int B, int C, CodecParams codec, const double *prefix, const double *block_mass,
                                   const uint32_t *shot_block, const double *rin, uint64_t nshots, uint64_t *out,
                                   cudaStream_t stream);
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
// *out = non-zero when every one of the nb blocks is stored, else 0.
// *out (set to 1 by the caller beforehand) is cleared when a block of the
// mask is not stored.
cudaError_t launch_mask_full(const uint8_t *mask, uint32_t nb, uint32_t *out, cudaStream_t stream);
// Up to four device arrays of 64-bit words gathered into one buffer.
struct ReadbackList {
    const unsigned long long *src[4];
    size_t words[4];
    int n;
};
cudaError_t launch_readback(const ReadbackList &l, unsigned long long *dst, cudaStream_t stream);
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

// Imported stores: headers of the chunks of unstored blocks set to zero.
cudaError_t launch_zero_unstored_headers(ChunkMeta *meta, const uint8_t *mask, uint64_t nchunks, int cshift,
                                         cudaStream_t stream);

// ---- chunk exchange between ranks (qubit swap across the rank boundary)
// The half of a store whose chunk-index bit `bit` (= qubit - C) equals v, in
// the order of the other index bits ("half index" k).  Export packs its
// headers (offsets relative to the packed payload, width 0 and base 0 for
// chunks of unstored blocks, flag 1 for stored ones) and payloads; import
// writes received chunks to the same positions of another store.
struct HalfChunks {
    int32_t bit;          // chunk-index bit of the exchanged qubit
    uint32_t value;       // the half: chunks whose bit equals value
    int32_t cshift;       // B - C: chunk index >> cshift = block
    int32_t C;
    uint64_t nhalf;       // chunks in the half
};
// sizes[k] = payload bytes of half chunk k (0 for unstored blocks), flags[k] = stored
cudaError_t launch_half_sizes(const HalfChunks &h, const ChunkMeta *meta, const uint8_t *mask, uint64_t *sizes,
                              uint8_t *flags, cudaStream_t stream);
// In-place exclusive scan of n sizes; *total receives their sum.  scratch:
// half_scan_scratch_words(n) 8-byte words.
uint64_t half_scan_scratch_words(uint64_t n);
cudaError_t launch_half_scan(uint64_t *sizes, uint64_t n, uint64_t *scratch, uint64_t *total, cudaStream_t stream);
// Packed headers and payloads of the half (offsets[k]: exclusive scan of
// sizes); headers go to out_meta[k], or with scatter to out_meta[chunk] (a
// store's own header array: the compaction of the half a rank keeps).
// Chunks of unstored blocks get zero headers.
cudaError_t launch_half_pack(const HalfChunks &h, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *flags,
                             const uint64_t *offsets, ChunkMeta *out_meta, uint32_t *out_payload, bool scatter,
                             cudaStream_t stream);
// Import: received headers written to their chunks with offsets rebased by
// base (bytes into the arena), their blocks marked stored (a block-level
// qubit: the block's stored flag is the received one).
cudaError_t launch_half_unpack(const HalfChunks &h, const ChunkMeta *in_meta, const uint8_t *in_flags, uint64_t base,
                               ChunkMeta *meta, uint8_t *mask, cudaStream_t stream);
// *bad = 1 when a received stored chunk's header is out of range.
cudaError_t launch_half_check(const HalfChunks &h, const ChunkMeta *in_meta, const uint8_t *in_flags,
                              uint64_t payload_bytes_total, int32_t *bad, cudaStream_t stream);
// block_bytes[b] = stored ? sum over its chunks of payload + 16 : 0.
cudaError_t launch_block_bytes(const ChunkMeta *meta, const uint8_t *mask, uint32_t nb, int cshift, int C,
                               unsigned long long *block_bytes, cudaStream_t stream);

// One CTA arms an mbarrier that nothing completes and runs the bounded wait
// of the staged kernels with `tries` tries; *gave_up = 1 when it gave up.
cudaError_t launch_bounded_wait_selftest(uint32_t tries, int32_t *gave_up, cudaStream_t stream);

int sm_count();

}  // namespace qs
