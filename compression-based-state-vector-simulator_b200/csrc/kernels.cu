// Device code of the compressed state-vector engine (sm_100a).
//
// The hot path is pass_kernel: one fused pass of a circuit stage over the
// HBM-resident compressed store.  It replaces, for every active group of the
// stage, the reference's chain H2D -> Bitcomp decode + inverse compander ->
// one kernel per gate per block pair -> zero check -> compander + Bitcomp
// encode -> D2H (src/cppsim/compressed_state_cuda.cu:143-381, kernels
// :392-811, compand_kernel.cuh:5-30, cuda_complex_helper.cuh:96-106).
//
// Work unit: a tile = 2^j chunks (2^C amplitudes each) whose chunk indices
// differ exactly in the pass's tile qubits, so every gate of the pass that
// mixes amplitudes acts inside one tile.  A CTA decodes the tile's chunks
// into shared memory (one warp per chunk, coalesced 128-byte payload rows),
// applies the pass's gates in shared memory, re-quantises, reserves output
// space for the whole tile with one atomicAdd on the arena's bump counter
// and writes the packed chunks back with coalesced stores.
#include <cstdio>
#include <climits>
#include <cstdlib>
#include <map>
#include <mutex>

#include "codec.cuh"
#include "internal.h"

namespace qs {

namespace {

template <typename R> struct Cplx;
template <> struct Cplx<float> { using T = float2; };
template <> struct Cplx<double> { using T = double2; };

template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
    T r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

template <typename T>
__device__ __forceinline__ T cfma(T a, T b, T c) {  // a*b + c
    T r;
    r.x = fma(a.x, b.x, fma(-a.y, b.y, c.x));
    r.y = fma(a.x, b.y, fma(a.y, b.x, c.y));
    return r;
}

template <typename T, typename R>
__device__ __forceinline__ T make_c(double re, double im) {
    T r;
    r.x = (R)re;
    r.y = (R)im;
    return r;
}

__device__ __forceinline__ uint64_t insert_zero_bits(uint64_t x, const int32_t *pos, int cnt) {
    for (int s = 0; s < cnt; ++s) {
        const int t = pos[s];
        const uint64_t lo = x & ((uint64_t(1) << t) - 1);
        x = ((x >> t) << (t + 1)) | lo;
    }
    return x;
}

__device__ __forceinline__ uint64_t deposit_bits(uint32_t c, const int32_t *pos, int cnt) {
    uint64_t r = 0;
    for (int s = 0; s < cnt; ++s) r |= uint64_t((c >> s) & 1u) << pos[s];
    return r;
}

// ------------------------------------------------------------ tile layout
// Element e of a tile lives at shared-memory slot swz(e) = e ^ ((e >> S1) & m):
// an XOR of the low S1 bits with the next ones, so that a warp whose lanes
// differ in any set of tile bits spreads over the banks.  m is limited to
// bits below the chunk size, so an element never leaves its chunk's region.
template <typename R> struct Layout;
template <> struct Layout<double> { static constexpr int S1 = 3; };
template <> struct Layout<float> { static constexpr int S1 = 4; };

template <typename R>
__host__ __device__ __forceinline__ int swizzle_mask(int C) {
    const int room = C - Layout<R>::S1;  // chunk bits above S1
    const int bits = room < Layout<R>::S1 ? (room > 0 ? room : 0) : Layout<R>::S1;
    return (1 << bits) - 1;
}

template <typename R>
__device__ __forceinline__ int swz(int e, int m) {
    return e ^ ((e >> Layout<R>::S1) & m);
}

// ------------------------------------------------------------ register gates
// v[s], s < NS = 2^RB, holds the tile element whose sweep bits equal s.
template <int NS, int K, typename T>
__device__ __forceinline__ void r_2x2(T (&v)[NS], T e0, T e1, T e2, T e3) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if ((s >> K) & 1) continue;
        const T a = v[s], b = v[s | (1 << K)];
        v[s] = cfma(e0, a, cmul(e1, b));
        v[s | (1 << K)] = cfma(e2, a, cmul(e3, b));
    }
}

template <int NS, int K, typename T>
__device__ __forceinline__ void r_diag2(T (&v)[NS], T d0, T d1) {
#pragma unroll
    for (int s = 0; s < NS; ++s) v[s] = cmul(((s >> K) & 1) ? d1 : d0, v[s]);
}

template <int NS, int KA, int KB, typename T>
__device__ __forceinline__ void r_4x4(T (&v)[NS], const T *__restrict__ m) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (((s >> KA) & 1) || ((s >> KB) & 1)) continue;
        const int i0 = s, i1 = s | (1 << KA), i2 = s | (1 << KB), i3 = s | (1 << KA) | (1 << KB);
        const T x0 = v[i0], x1 = v[i1], x2 = v[i2], x3 = v[i3];
        T o[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            T acc = cmul(m[4 * r + 0], x0);
            acc = cfma(m[4 * r + 1], x1, acc);
            acc = cfma(m[4 * r + 2], x2, acc);
            acc = cfma(m[4 * r + 3], x3, acc);
            o[r] = acc;
        }
        v[i0] = o[0];
        v[i1] = o[1];
        v[i2] = o[2];
        v[i3] = o[3];
    }
}

template <int NS, int KA, int KB, typename T>
__device__ __forceinline__ void r_diag4(T (&v)[NS], T d0, T d1, T d2, T d3) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int k = ((s >> KA) & 1) | (((s >> KB) & 1) << 1);
        v[s] = cmul(k == 0 ? d0 : (k == 1 ? d1 : (k == 2 ? d2 : d3)), v[s]);
    }
}

template <typename T>
__device__ __forceinline__ T c_one() { T r; r.x = 1; r.y = 0; return r; }

template <int NS, int K, typename T>
__device__ __forceinline__ void r_half2(T (&v)[NS], T d1) {
#pragma unroll
    for (int s = 0; s < NS; ++s)
        if ((s >> K) & 1) v[s] = cmul(d1, v[s]);
}

template <int NS, int KA, int KB, typename T>
__device__ __forceinline__ void r_half4(T (&v)[NS], T d1, T d2, T d3) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int k = ((s >> KA) & 1) | (((s >> KB) & 1) << 1);
        if (k) v[s] = cmul(k == 1 ? d1 : (k == 2 ? d2 : d3), v[s]);
    }
}

template <int NS, int K, typename T>
__device__ __forceinline__ void r_x(T (&v)[NS]) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if ((s >> K) & 1) continue;
        const T t = v[s];
        v[s] = v[s | (1 << K)];
        v[s | (1 << K)] = t;
    }
}

template <int NS, int KA, int KB, typename T>
__device__ __forceinline__ void r_swap(T (&v)[NS]) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (((s >> KA) & 1) || ((s >> KB) & 1)) continue;
        const T t = v[s | (1 << KA)];
        v[s | (1 << KA)] = v[s | (1 << KB)];
        v[s | (1 << KB)] = t;
    }
}

// One register op on a group (codes in internal.h).  z collects the group's
// scalar factors and is applied when the group is stored.
template <int RB, typename T>
__device__ __forceinline__ void apply_rop(T (&v)[1 << RB], T &z, T &zh, int code, const T *__restrict__ m) {
    constexpr int NS = 1 << RB;
#define QS_K(BASE, K, ...) \
    case BASE + K:         \
        if constexpr (K < RB) { __VA_ARGS__; } \
        break;
#define QS_P(BASE, A, B, ...) \
    case BASE + (A) * 8 + (B): \
        if constexpr ((A) < RB && (B) < RB) { __VA_ARGS__; } \
        break;
#define QS_ALLK(BASE, F) F(BASE, 0) F(BASE, 1) F(BASE, 2) F(BASE, 3) F(BASE, 4)
#define QS_ALLP(BASE, F) F(BASE, 0, 1) F(BASE, 0, 2) F(BASE, 0, 3) F(BASE, 0, 4) F(BASE, 1, 2) \
    F(BASE, 1, 3) F(BASE, 1, 4) F(BASE, 2, 3) F(BASE, 2, 4) F(BASE, 3, 4)
#define QS_D2(B, K) QS_K(B, K, r_diag2<NS, K>(v, m[0], m[1]))
#define QS_D2H(B, K) QS_K(B, K, r_half2<NS, K>(v, m[0]))
#define QS_D2HP(B, K) QS_K(B, K, r_half2<NS, K>(v, cmul(zh, m[0])); zh = c_one<T>())
#define QS_M2(B, K) QS_K(B, K, r_2x2<NS, K>(v, m[0], m[1], m[2], m[3]))
#define QS_X(B, K) QS_K(B, K, r_x<NS, K>(v))
#define QS_D4(B, A, C) QS_P(B, A, C, r_diag4<NS, A, C>(v, m[0], m[1], m[2], m[3]))
#define QS_D4H(B, A, C) QS_P(B, A, C, r_half4<NS, A, C>(v, m[0], m[1], m[2]))
#define QS_M4(B, A, C) QS_P(B, A, C, r_4x4<NS, A, C>(v, m))
#define QS_SW(B, A, C) QS_P(B, A, C, r_swap<NS, A, C>(v))
    switch (code) {
        case OPC_SCALAR: z = cmul(z, m[0]); break;
        case OPC_ACC: zh = cmul(zh, m[0]); break;
        QS_ALLK(OPC_D2, QS_D2)
        QS_ALLK(OPC_D2H, QS_D2H)
        QS_ALLK(OPC_D2HP, QS_D2HP)
        QS_ALLK(OPC_M2, QS_M2)
        QS_ALLK(OPC_X, QS_X)
        QS_ALLP(OPC_D4, QS_D4)
        QS_ALLP(OPC_D4H, QS_D4H)
        QS_ALLP(OPC_M4, QS_M4)
        QS_ALLP(OPC_SWAP, QS_SW)
        default: break;
    }
#undef QS_K
#undef QS_P
#undef QS_ALLK
#undef QS_ALLP
#undef QS_D2
#undef QS_D2H
#undef QS_D2HP
#undef QS_M2
#undef QS_X
#undef QS_D4
#undef QS_D4H
#undef QS_M4
#undef QS_SW
}

// Variant index of an op for a group with word W (selector bits of W).
__device__ __forceinline__ uint32_t rop_variant(const ROp &o, uint32_t W) {
    uint32_t var = 0;
    if (o.sel[0] & kSelRuns) {
        const uint32_t a = o.sel[0] & 31u, la = o.sel[1], b = o.sel[2], lb = o.sel[3];
        return ((W >> a) & ((1u << la) - 1u)) | (((W >> b) & ((1u << lb) - 1u)) << la);
    }
    if (o.nsel) {
#pragma unroll
        for (int j = 0; j < 4; ++j) var |= ((W >> o.sel[j]) & 1u) << j;
        if (o.nsel > 4) {
#pragma unroll
            for (int j = 4; j < kMaxSel; ++j) var |= ((W >> o.sel[j]) & 1u) << j;
        }
    }
    return var;
}

// Outer selector word of a tile whose element 0 is global amplitude base_amp.
__device__ __forceinline__ uint32_t outer_word(uint64_t base_amp, const int8_t *outer_q, int nouter) {
    uint32_t w = 0;
    for (int i = 0; i < nouter; ++i) w |= (uint32_t)((base_amp >> outer_q[i]) & 1u) << i;
    return w;
}

// Apply every sweep of a pass to a tile of 2^nb elements.  ow is the tile's
// outer selector word.  For complex64 they are a separate (not inlined)
// function: it gets its own register allocation, apart from the codec phases
// of the pass kernel, which measured faster; complex128 keeps them inlined.
template <typename R, int RB>
__device__ __forceinline__ void tile_sweeps_body(typename Cplx<R>::T *tile, int nb, int swm,
                                                 const Sweep *__restrict__ sweeps, int nsweeps,
                                                 const ROp *__restrict__ ops,
                                                 const typename Cplx<R>::T *__restrict__ pool, uint32_t ow);
template <typename R, int RB>
__device__ __noinline__ void tile_sweeps_call(typename Cplx<R>::T *tile, int nb, int swm, const Sweep *__restrict__ sweeps,
                            int nsweeps, const ROp *__restrict__ ops, const typename Cplx<R>::T *__restrict__ pool,
                            uint32_t ow) { tile_sweeps_body<R, RB>(tile, nb, swm, sweeps, nsweeps, ops, pool, ow); }
template <typename R, int RB>
__device__ __forceinline__ void tile_sweeps(typename Cplx<R>::T *tile, int nb, int swm, const Sweep *__restrict__ sweeps,
                            int nsweeps, const ROp *__restrict__ ops, const typename Cplx<R>::T *__restrict__ pool,
                            uint32_t ow) {
    if constexpr (sizeof(R) == 4) tile_sweeps_call<R, RB>(tile, nb, swm, sweeps, nsweeps, ops, pool, ow);
    else tile_sweeps_body<R, RB>(tile, nb, swm, sweeps, nsweeps, ops, pool, ow);
}
template <typename R, int RB>
__device__ __forceinline__ void tile_sweeps_body(typename Cplx<R>::T *tile, int nb, int swm, const Sweep *__restrict__ sweeps,
                            int nsweeps, const ROp *__restrict__ ops, const typename Cplx<R>::T *__restrict__ pool,
                            uint32_t ow) {
    using T = typename Cplx<R>::T;
    constexpr int NS = 1 << RB;
    const int groups = 1 << (nb - RB);
    const uint32_t wo = ow << nb;
    for (int w = 0; w < nsweeps; ++w) {
        const Sweep sw = sweeps[w];
        int sb[RB], bm[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            sb[k] = sw.sbits[k];
            bm[k] = 1 << sb[k];
        }
        // offset of group element s: the OR of the masks of its set bits (s is
        // a compile-time index, so each offset is a few ORs, no table)
        auto off = [&](int s) {
            int o = 0;
#pragma unroll
            for (int k = 0; k < RB; ++k)
                if ((s >> k) & 1) o |= bm[k];
            return o;
        };
        for (int grp = threadIdx.x; grp < groups; grp += blockDim.x) {
            int base = grp;
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                const int t = sb[k];
                base = ((base >> t) << (t + 1)) | (base & ((1 << t) - 1));
            }
            const uint32_t W = (uint32_t)base | wo;
            T v[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) v[s] = tile[swz<R>(base | off(s), swm)];
            T z = c_one<T>(), zh = c_one<T>();
            for (int k = sw.g0; k < sw.g1; ++k) {
                const ROp o = ops[k];
                apply_rop<RB>(v, z, zh, o.code, pool + o.mat + rop_variant(o, W) * o.vstride);
            }
            if (z.x != R(1) || z.y != R(0)) {
#pragma unroll
                for (int s = 0; s < NS; ++s) v[s] = cmul(z, v[s]);
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) tile[swz<R>(base | off(s), swm)] = v[s];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ chunk codec
// Per-warp decode of one chunk into comp[lane + 32 i] (i < per_lane).
struct LinearSlot {
    __device__ __forceinline__ int operator()(int c) const { return c; }
};

// Component c of chunk `chunk` inside a swizzled tile.
template <typename R>
struct TileSlot {
    int elem0, swm;
    __device__ __forceinline__ int operator()(int c) const { return 2 * swz<R>(elem0 + (c >> 1), swm) + (c & 1); }
};

// A quantised code held in a tile slot of type R (its bit pattern; only
// moved, never used in arithmetic), for passes that move amplitudes
// without changing them.  quantise(dequantise(c)) == c for every code, so
// moving codes gives the same store as moving values.
__device__ __forceinline__ float code_as_value(int32_t c, float) { return __int_as_float(c); }
__device__ __forceinline__ double code_as_value(int32_t c, double) { return __longlong_as_double((long long)c); }
__device__ __forceinline__ int32_t value_as_code(float v) { return __float_as_int(v); }
__device__ __forceinline__ int32_t value_as_code(double v) { return (int32_t)__double_as_longlong(v); }

// Words of the per-warp staging area of decode_chunk: one row more than a
// chunk can use, so that the look-ahead word of the last row stays inside.
constexpr int kStageWords = (kMaxPerLane + 1) * 32;

// Start the asynchronous copy of a chunk's payload (rows x 128 contiguous
// bytes, 128-byte aligned) into a warp's staging buffer: 16-byte cp.async
// copies, no registers, one commit group per call (empty for width 0).
__device__ __forceinline__ void issue_payload(const uint32_t *__restrict__ arena, const ChunkMeta md, int per_lane,
                                              uint32_t *dst, int lane) {
    const int rows = (int)(((uint32_t)per_lane * md.width + 31) >> 5);
    const uint32_t sdst = (uint32_t)__cvta_generic_to_shared(dst);
    const char *gsrc = reinterpret_cast<const char *>(arena + (md.offset >> 2));
    for (int off = lane * 16; off < rows * 128; off += 32 * 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sdst + off), "l"(gsrc + off) : "memory");
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Unpack a chunk whose payload is in the warp's staging buffer (the copy
// complete and visible to the warp): every element is extracted on its own
// (one funnel shift); a lane reads only its own words.
template <typename R, typename Slot = LinearSlot, bool kCodes = false>
__device__ __forceinline__ void unpack_chunk(const ChunkMeta md, int per_lane, CodecParams p, R *comp,
                                             const uint32_t *wstage, int lane, Slot slot = Slot()) {
    // a width above 32 never comes from a pass or a checked import; clamped so
    // that no header can make the unpack read past its chunk's staged rows
    const uint32_t w = md.width > 32 ? 32u : md.width;
    if (w == 0) {
        const R v = kCodes ? code_as_value(md.base, R()) : dequantize_hot(md.base, p, R());
        for (int i = 0; i < per_lane; ++i) comp[slot(lane + 32 * i)] = v;
        return;
    }
    const uint32_t mask = (w >= 32) ? 0xffffffffu : ((1u << w) - 1u);
#pragma unroll
    for (int i = 0; i < kMaxPerLane; ++i) {
        if (i < per_lane) {
            const uint32_t bit = (uint32_t)i * w, r = bit >> 5;
            const uint32_t u = __funnelshift_r(wstage[r * 32 + lane], wstage[(r + 1) * 32 + lane], bit & 31) & mask;
            const int32_t code = (int32_t)((uint32_t)md.base + u);
            comp[slot(lane + 32 * i)] = kCodes ? code_as_value(code, R()) : dequantize_hot(code, p, R());
        }
    }
}

// Per-warp decode of one chunk: copy its payload into the warp's staging
// area (one round trip to memory), then unpack it.
template <typename R, typename Slot = LinearSlot, bool kCodes = false>
__device__ __forceinline__ void decode_chunk(const uint32_t *__restrict__ arena, const ChunkMeta md,
                                             int per_lane, CodecParams p, R *comp, uint32_t *wstage,
                                             int lane, Slot slot = Slot()) {
    if (md.width != 0) {
        issue_payload(arena, md, per_lane, wstage, lane);
        cp_async_wait<0>();
        __syncwarp();
    }
    unpack_chunk<R, Slot, kCodes>(md, per_lane, p, comp, wstage, lane, slot);
}

// Per-warp quantisation of one chunk held in comp[]: codes overwrite the
// chunk's own shared memory as int32.  Returns
// base/width/non-zero flag (valid in every lane).
template <typename R, typename Slot = LinearSlot, bool kCodes = false>
__device__ __forceinline__ void quantize_chunk(R *comp, int per_lane, CodecParams p, bool exact_zero,
                                               int lane, int32_t *base_out, uint32_t *width_out,
                                               bool *nz_out, Slot slot = Slot(), int32_t *codes = nullptr) {
    if (codes == nullptr) codes = reinterpret_cast<int32_t *>(comp);
    int32_t lo = INT_MAX, hi = INT_MIN;
    bool nz = false;
    // four quarters, to cut the live values: the code of component c is 4
    // bytes at offset 4c of the chunk's region and its value lies at or after
    // that offset, so the codes of a quarter overwrite only values already read
    constexpr int H = kMaxPerLane / 4;
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        R v[H];
#pragma unroll
        for (int i = 0; i < H; ++i)
            if (h * H + i < per_lane) v[i] = comp[slot(lane + 32 * (h * H + i))];
        __syncwarp();
#pragma unroll
        for (int i = 0; i < H; ++i) {
            if (h * H + i < per_lane) {
                const int32_t q = kCodes ? value_as_code(v[i]) : quantize_hot(v[i], p);
                codes[lane + 32 * (h * H + i)] = q;
                lo = min(lo, q);
                hi = max(hi, q);
                // code 0 is exactly the value 0
                nz |= (exact_zero && !kCodes) ? (v[i] != R(0)) : (q != 0);
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    nz = __any_sync(0xffffffffu, nz);
    __syncwarp();
    *base_out = lo;
    *width_out = bit_length((uint32_t)((int64_t)hi - (int64_t)lo));
    *nz_out = nz;
}

// Per-warp packing of int32 codes[lane + 32 i] to dst (layout in codec.cuh).
__device__ __forceinline__ void pack_chunk(const int32_t *codes, int per_lane, int32_t base, uint32_t w,
                                           uint32_t *__restrict__ dst, int lane) {
    if (w == 0) return;
    uint64_t buf = 0;
    uint32_t nbits = 0, r = 0;
    for (int i = 0; i < per_lane; ++i) {
        const uint32_t u = (uint32_t)(codes[lane + 32 * i] - base);
        buf |= (uint64_t)u << nbits;
        nbits += w;
        if (nbits >= 32) {
            __stcs(dst + r * 32 + lane, (uint32_t)buf);
            ++r;
            buf >>= 32;
            nbits -= 32;
        }
    }
    if (nbits > 0) __stcs(dst + r * 32 + lane, (uint32_t)buf);
}

__device__ __forceinline__ uint64_t apply_perm(const ChunkPerm &p, uint64_t c) {
    uint64_t o = c & p.keep;
    for (int k = 0; k < p.nmove; ++k) o |= ((c >> p.src[k]) & 1ull) << p.dst[k];
    return o ^ p.flip;
}

size_t pass_smem_bytes(bool f64, int nb, int j) {
    const size_t tile = (f64 ? 16 : 8) << nb;
    const size_t stage = (size_t)(kSweepThreads / 32) * kStageWords * 4;
    const size_t tables = ((size_t)3 * 4 << j) + 8;
    const size_t offs = (size_t)8 << j;
    const size_t headers = sizeof(ChunkMeta) << j;
    return tile + stage + ((tables + 7) / 8) * 8 + offs + headers;
}

// ------------------------------------------------------------ diagonal Pauli sum
// tile[e] *= sum_t c_t (-1)^{|e & zt_t| + |base_amp & zo_t|}: the outer sign
// of each term is folded into its coefficient once per tile (s_dc, 2 doubles
// per term, written and read by the whole CTA between barriers).
template <typename R>
__device__ void tile_diag_sum(typename Cplx<R>::T *tile, int nb, int swm, const DiagSum &d, uint64_t base_amp,
                              double *s_dc) {
    using T = typename Cplx<R>::T;
    for (int t = threadIdx.x; t < d.nterms; t += blockDim.x) {
        const double sg = (__popcll(base_amp & d.terms[t].zo) & 1) ? -1.0 : 1.0;
        s_dc[2 * t] = sg * d.coefs[2 * t];
        s_dc[2 * t + 1] = sg * d.coefs[2 * t + 1];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < (1 << nb); e += blockDim.x) {
        double hr = 0.0, hi = 0.0;
        for (int t = 0; t < d.nterms; ++t) {
            const double sg = (__popc((uint32_t)e & d.terms[t].zt) & 1) ? -1.0 : 1.0;
            hr = fma(sg, s_dc[2 * t], hr);
            hi = fma(sg, s_dc[2 * t + 1], hi);
        }
        T &v = tile[swz<R>(e, swm)];
        const double vr = (double)v.x, vi = (double)v.y;
        v.x = (R)(hr * vr - hi * vi);
        v.y = (R)(hr * vi + hi * vr);
    }
    __syncthreads();
}

static_assert((kSweepThreads / 32) * kStageWords * 4 >= 2 * kMaxDiagTerms * sizeof(double),
              "the pass kernel's decode staging holds the diagonal-sum coefficients");

// ------------------------------------------------------------ pass kernel
// Whether a warp loads all its chunk headers at once and copies its next
// chunk's payload while it unpacks the current one (complex128, measured
// faster there), or loads headers four at a time and copies each payload
// just before unpacking it (complex64, measured faster there).
template <typename R>
constexpr bool kPrefetchDecode = sizeof(R) == 8;

// ------------------------------------------------------------ pass kernel
// kCodes: every op of the pass only moves amplitudes (X / SWAP register
// moves, chunk permutations), so the tile holds the quantised codes
// themselves and the pass skips dequantisation and quantisation.
// kHB: complex64 chunk headers loaded per warp batch (4 or 8).
// kC, kJ: the chunk log2 and the tile qubits above the chunk when known at
// compile time, 0 to read them from the args.
template <typename R, int RB, bool kCodes, int kHB, int kC, int kJ>
__global__ void __launch_bounds__(kSweepThreads, 3) pass_kernel(const PassArgs a) {
    using T = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long s_tile_off, s_next, s_slab_end;
    __shared__ int s_flag;
    __shared__ int32_t s_tq[kMaxTileQubits];
    __shared__ int8_t s_oq[kMaxOuterSel];
    if (threadIdx.x < kMaxTileQubits) s_tq[threadIdx.x] = a.tq[threadIdx.x];
    if (threadIdx.x < kMaxOuterSel) s_oq[threadIdx.x] = a.outer_q[threadIdx.x];
    if (threadIdx.x == 0) {
        s_next = 0;
        s_slab_end = 0;
    }
    __syncthreads();

    const int C = kC ? kC : a.C, j = kJ ? kJ : a.j, nb = C + j;
    const int nchunks = 1 << j;
    const int ncomp = 2 << C;
    const int per_lane = ncomp >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int blk_shift = a.B - C;
    const int swm = swizzle_mask<R>(C);

    T *tile = reinterpret_cast<T *>(smem);
    uint32_t *stage_all = reinterpret_cast<uint32_t *>(smem + (sizeof(T) << nb));
    uint32_t *wstage = stage_all + warp * kStageWords;
    int32_t *s_base = reinterpret_cast<int32_t *>(stage_all + nwarps * kStageWords);
    uint32_t *s_width = reinterpret_cast<uint32_t *>(s_base + nchunks);
    uint32_t *s_nz = s_width + nchunks;
    unsigned long long *s_off = reinterpret_cast<unsigned long long *>(
        reinterpret_cast<unsigned char *>(s_base) + ((((size_t)3 * 4 << j) + 8 + 7) / 8) * 8);
    ChunkMeta *s_md = reinterpret_cast<ChunkMeta *>(s_off + nchunks);

    unsigned long long rd = 0, wr = 0, ntiles = 0;

    for (uint64_t tile_id = blockIdx.x; tile_id < a.n_tiles; tile_id += gridDim.x) {
        const uint64_t chunk_base = insert_zero_bits(tile_id, s_tq, j);
        const uint64_t block0 = chunk_base >> blk_shift;
        if (!a.group_active[a.block_to_group[block0]]) continue;  // uniform in the CTA
        if (threadIdx.x == 0) s_flag = *reinterpret_cast<volatile int32_t *>(a.error);
        __syncthreads();
        if (s_flag) break;
        ++ntiles;

        if constexpr (!kPrefetchDecode<R>) {
            // ---- decode: the headers of kHB of the warp's chunks are
            // loaded together, then the chunks are unpacked one by one
            constexpr int HB = kHB;
            for (int c0 = warp; c0 < nchunks; c0 += HB * nwarps) {
                ChunkMeta md[HB];
                bool zero[HB];
#pragma unroll
                for (int b = 0; b < HB; ++b) {
                    const int c = c0 + b * nwarps;
                    md[b] = ChunkMeta{0, 0, 0};
                    zero[b] = true;
                    if (c < nchunks) {
                        const uint64_t chunk = chunk_base | deposit_bits((uint32_t)c, s_tq, j);
                        if (!a.first_pass || a.mask[chunk >> blk_shift]) {
                            md[b] = a.meta_in[chunk];
                            zero[b] = false;
                        }
                    }
                }
#pragma unroll
                for (int b = 0; b < HB; ++b) {
                    const int c = c0 + b * nwarps;
                    if (c >= nchunks) break;
                    R *comp = reinterpret_cast<R *>(tile) + (size_t)c * ncomp;
                    if (zero[b]) {
                        for (int i = 0; i < per_lane; ++i) comp[lane + 32 * i] = R(0);
                        continue;
                    }
                    decode_chunk<R, TileSlot<R>, kCodes>(a.arena_in, md[b], per_lane, a.codec,
                                                         reinterpret_cast<R *>(tile), wstage, lane,
                                                         TileSlot<R>{c << C, swm});
                    if (lane == 0) rd += payload_bytes(C, md[b].width) + sizeof(ChunkMeta);
                }
            }
        } else {
            // ---- decode.  A warp's lanes load the headers of all of the
            // warp's chunks at once (a chunk of a zero block reads as width 0,
            // base 0: zeros).  The warp then walks its chunks and copies the
            // next chunk's payload with cp.async while it unpacks the current
            // one; the two payload buffers are the warp's staging area and
            // the tile region of the warp's last chunk, which nothing uses
            // until that chunk is unpacked.
            for (int c = warp + lane * nwarps; c < nchunks; c += 32 * nwarps) {
                ChunkMeta md{0, 0, 0};
                const uint64_t chunk = chunk_base | deposit_bits((uint32_t)c, s_tq, j);
                if (!a.first_pass || a.mask[chunk >> blk_shift]) {
                    md = a.meta_in[chunk];
                    rd += payload_bytes(C, md.width) + sizeof(ChunkMeta);
                }
                s_md[c] = md;
            }
            __syncwarp();
            const int m = warp < nchunks ? (nchunks - warp + nwarps - 1) / nwarps : 0;
            if (m > 0) {
                uint32_t *bufR = reinterpret_cast<uint32_t *>(reinterpret_cast<R *>(tile) +
                                                              (size_t)(warp + (m - 1) * nwarps) * ncomp);
                issue_payload(a.arena_in, s_md[warp], per_lane, wstage, lane);
                for (int i = 0; i < m; ++i) {
                    const int c = warp + i * nwarps;
                    uint32_t *cur = (i < m - 1 && (i & 1)) ? bufR : wstage;
                    uint32_t *nxt = (i + 1 < m - 1 && ((i + 1) & 1)) ? bufR : wstage;
                    const bool pre = i + 1 < m && nxt != cur;
                    if (pre) {
                        issue_payload(a.arena_in, s_md[c + nwarps], per_lane, nxt, lane);
                        cp_async_wait<1>();
                    } else {
                        cp_async_wait<0>();
                    }
                    __syncwarp();
                    unpack_chunk<R, TileSlot<R>, kCodes>(s_md[c], per_lane, a.codec, reinterpret_cast<R *>(tile), cur,
                                                         lane, TileSlot<R>{c << C, swm});
                    __syncwarp();
                    if (i + 1 < m && !pre) issue_payload(a.arena_in, s_md[c + nwarps], per_lane, nxt, lane);
                }
            }
        }
        __syncthreads();

        // ---- gates
        tile_sweeps<R, RB>(tile, nb, swm, a.sweeps, a.nsweeps, a.ops, reinterpret_cast<const T *>(a.pool),
                           outer_word(chunk_base << C, s_oq, a.nouter));
        // the decode staging area is free here: it holds the tile's term coefficients
        if constexpr (!kCodes) {
            if (a.diag.nterms)
                tile_diag_sum<R>(tile, nb, swm, a.diag, chunk_base << C, reinterpret_cast<double *>(stage_all));
        }

        // ---- quantise (codes replace values in shared memory)
        for (int c = warp; c < nchunks; c += nwarps) {
            R *comp = reinterpret_cast<R *>(tile) + (size_t)c * ncomp;
            int32_t base;
            uint32_t width;
            bool nz;
            quantize_chunk<R, TileSlot<R>, kCodes>(reinterpret_cast<R *>(tile), per_lane, a.codec, a.exact_zero != 0,
                                                   lane, &base, &width, &nz, TileSlot<R>{c << C, swm},
                                                   reinterpret_cast<int32_t *>(comp));
            if (lane == 0) {
                s_base[c] = base;
                s_width[c] = width;
                s_nz[c] = nz ? 1u : 0u;
            }
        }
        __syncthreads();

        // ---- reserve the tile's output bytes with one atomic: warp 0 scans
        // the chunk sizes (each lane a run of consecutive chunks)
        if (warp == 0) {
            const int per = (nchunks + 31) >> 5;
            const int c0 = lane * per;
            unsigned long long mine = 0;
            for (int c = c0; c < c0 + per && c < nchunks; ++c) mine += payload_bytes(C, s_width[c]);
            unsigned long long incl = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            unsigned long long run = incl - mine;
            for (int c = c0; c < c0 + per && c < nchunks; ++c) {
                s_off[c] = run;
                run += payload_bytes(C, s_width[c]);
            }
            const unsigned long long total = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == 0) {
                // the tile goes at the CTA's next free byte of its current
                // slab; one that does not fit takes a new slab of a.slab
                // bytes (or exactly its own size) from the arena, so most
                // tiles reserve without touching the shared counter
                unsigned long long off = s_next;
                s_flag = 0;
                if (a.slab == 0 || off + total > s_slab_end) {
                    const unsigned long long want = total > a.slab ? total : a.slab;
                    off = atomicAdd(a.bump, want);
                    if (off + want > a.capacity) {
                        atomicExch(a.error, 1);
                        s_flag = 1;
                    }
                    s_slab_end = off + want;
                }
                s_tile_off = off;
                s_next = off + total;
                wr += total + (unsigned long long)nchunks * sizeof(ChunkMeta);
            }
        }
        __syncthreads();
        if (s_flag) break;

        // ---- pack and store
        for (int c = warp; c < nchunks; c += nwarps) {
            const uint64_t chunk = apply_perm(a.perm, chunk_base | deposit_bits((uint32_t)c, s_tq, j));
            const int32_t *codes = reinterpret_cast<const int32_t *>(reinterpret_cast<R *>(tile) + (size_t)c * ncomp);
            const unsigned long long off = s_tile_off + s_off[c];
            const uint32_t w = s_width[c];
            pack_chunk(codes, per_lane, s_base[c], w, a.arena_out + (off >> 2), lane);
            if (lane == 0) {
                ChunkMeta md;
                md.offset = off;
                md.base = s_base[c];
                md.width = w;
                a.meta_out[chunk] = md;
                if (a.final_pass) {
                    const uint64_t blk = chunk >> blk_shift;
                    if (s_nz[c]) atomicOr(&a.block_nz[blk], 1u);
                    atomicAdd(&a.block_bytes[blk], (unsigned long long)(payload_bytes(C, w) + sizeof(ChunkMeta)));
                }
            }
        }
        __syncthreads();
    }
    if (rd) atomicAdd(&a.stats[0], rd);
    if (threadIdx.x == 0) {
        if (wr) atomicAdd(&a.stats[1], wr);
        if (ntiles) atomicAdd(&a.stats[2], ntiles);
    }
}

// ------------------------------------------------------------ staged pass kernel
// The same fused pass as pass_kernel, restructured so that no global-memory
// latency sits on a tile's critical path:
//   * persistent CTAs of kStagedThreads threads walk their tiles in order;
//     while a CTA works on tile t, the compressed payload of its next tile is
//     already streaming into a shared-memory double buffer with 1-D bulk
//     asynchronous copies (cp.async.bulk, one per chunk, completion counted
//     in bytes on an mbarrier), and the chunk headers of the tile after that
//     with 16-byte cp.async copies;
//   * which blocks belong to an active group and which were stored at the
//     start of the stage are read once per CTA into shared-memory bitmasks;
//   * the error flag is loaded at the start of a tile and tested only at the
//     tile's output reservation.
// Decode, sweeps, quantisation, reservation and packing are pass_kernel's.
// The copies read this GPU's own memory only (no cluster multicast).
constexpr int kStagedThreads = 256;
// Blocks whose activity / stored bits are kept in shared memory (two bitmasks
// of this many bits); passes over more blocks read them from global memory.
constexpr uint32_t kMaxSmemBlocks = 1u << 16;
// Iterations of a bounded mbarrier wait (each try_wait itself suspends for a
// while before it returns false).
constexpr uint32_t kMbarSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of `bar` with the given parity to complete; false when
// it has not after `tries` tries.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t tries = kMbarSpinLimit) {
    for (uint32_t i = 0; i < tries; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// The bounded wait's give-up path, exercised without any copy: thread 0
// arms an mbarrier for 16 bytes that nothing will deliver and waits at most
// `tries` times; *gave_up = 1 when the wait returned false (as it must), 0
// otherwise.  No asynchronous operation targets the barrier, so the CTA
// invalidates it and exits cleanly.
__global__ void bounded_wait_selftest_kernel(uint32_t tries, int32_t *gave_up) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, 16);
        const bool done = mbar_wait_bounded(&bar, 0, tries);
        mbar_inval(&bar);
        *gave_up = done ? 0 : 1;
    }
}

// 1-D bulk copy global -> this CTA's shared memory, completion (in bytes) on
// `bar`.  Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// Shared-memory layout of staged_pass_kernel (byte offsets; every region
// 128-byte aligned).
struct StagedLayout {
    size_t tile, buf0, buf1, hdr0, hdr1, poff0, poff1, base, width, nz, off, act, sto;
    size_t dense_a, dense_b, dense_dep;  // dense k-qubit passes only
    size_t total;
};

__host__ __device__ inline size_t align128(size_t x) { return (x + 127) / 128 * 128; }

// stage_bytes: one tile's largest payload (every chunk at width 32) plus one
// 128-byte row read ahead by the last chunk's unpack.
__host__ __device__ inline size_t staged_stage_bytes(int C, int j) {
    return ((size_t)1 << j) * payload_bytes(C, 32) + 128;
}

// Dense k-qubit passes add: complex64, the tile as the realified tcgen05 A
// operand (hi and lo parts, 2 x 4 x 2^(nb+1) bytes) and the gate operand (hi
// and lo, 2 x 4 x 2^(2k+2) bytes); complex128, the gate matrix (16 x
// 2^(2k) bytes); both, the tile offsets of the gate's 2^k patterns.
__host__ __device__ inline StagedLayout staged_layout(bool f64, int C, int j, uint32_t mask_words, int dense_k = 0) {
    StagedLayout L{};
    const size_t nch = (size_t)1 << j;
    size_t o = 0;
    L.tile = o;  o += align128((f64 ? 16 : 8) << (C + j));
    const size_t stage = align128(staged_stage_bytes(C, j));
    L.buf0 = o;  o += stage;
    L.buf1 = o;  o += stage;
    L.hdr0 = o;  o += align128(sizeof(ChunkMeta) * nch);
    L.hdr1 = o;  o += align128(sizeof(ChunkMeta) * nch);
    L.poff0 = o; o += align128(4 * nch);
    L.poff1 = o; o += align128(4 * nch);
    L.base = o;  o += align128(4 * nch);
    L.width = o; o += align128(4 * nch);
    L.nz = o;    o += align128(4 * nch);
    L.off = o;   o += align128(8 * nch);
    L.act = o;   o += align128(4 * (size_t)mask_words);
    L.sto = o;   o += align128(4 * (size_t)mask_words);
    if (dense_k > 0) {
        if (!f64) {
            L.dense_a = o; o += align128((size_t)2 * 4 * ((size_t)2 << (C + j)));
            L.dense_b = o; o += align128((size_t)2 * 4 * ((size_t)4 << (2 * dense_k)));
        } else {
            L.dense_b = o; o += align128((size_t)16 << (2 * dense_k));
        }
        L.dense_dep = o; o += align128(4 * ((size_t)1 << dense_k));
    }
    L.total = o;
    return L;
}

// ------------------------------------------------------------ dense k-qubit gate over a tile
// tcgen05 building blocks (sm_100a): shared-memory operand descriptors,
// the kind::tf32 MMA, its commit to an mbarrier, TMEM allocation and loads.

// Descriptor of a K-major, unswizzled operand (dense_k_operand_offset) whose
// first element is at shared address saddr: start >> 4 in bits [0, 14),
// leading byte offset (128: the next 4 columns) >> 4 in [16, 30), stride
// byte offset (kcols * 32: the next 8 rows) >> 4 in [32, 46), descriptor
// version 1 at bit 46, layout type 0 (no swizzle) in bits [61, 64).
__device__ __forceinline__ uint64_t umma_kmajor_desc(uint32_t saddr, uint32_t kcols) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)(((kcols * 32u) >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::tf32, FP32 accumulation, both operands
// K-major: D format F32 (1) in bits [4, 6), A and B format TF32 (2) in
// [7, 10) and [10, 13), N >> 3 in [17, 23), M >> 4 in [24, 29).
__host__ __device__ inline uint32_t umma_tf32_idesc(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n"
        "}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// 16 consecutive 32-bit columns of this warp's 32 TMEM lanes (lane = thread)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// x rounded to tf32 (10 mantissa bits, round to nearest, ties away)
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// TMEM columns of the dense accumulator: 2^(5-k) blocks of 128 rows x
// 2^(k+1) FP32 columns = 64 columns for every k of a 2^12 tile.
constexpr uint32_t kDenseTmemCols = 64;

// Tile bit patterns: dep[r] = tile offset of gate pattern r (matrix bit i
// at pos[i]); base of row o = o deposited into the other tile bits.
__device__ __forceinline__ uint32_t dense_row_base(uint32_t o, uint32_t gmask, int nb) {
    uint32_t b = 0;
    for (int t = 0, i = 0; t < nb; ++t) {
        if ((gmask >> t) & 1u) continue;
        b |= ((o >> i) & 1u) << t;
        ++i;
    }
    return b;
}

// complex64: y = G x for every column of the tile on the tensor cores.
// aop: the A operand area (hi part, then lo part), bop: the gate operand
// (hi, lo), dep: pattern offsets, d_tmem: the accumulator, bar: the MMA
// mbarrier with its phase parity.  Returns false when the MMAs did not
// complete within the bounded wait.
__device__ bool tile_dense_k_tc(float2 *tile, int nb, int swm, int k, const int32_t *dep, uint32_t gmask,
                                float *aop, const float *bop, uint32_t d_tmem, uint64_t *bar, uint32_t parity) {
    const int K = 1 << k;              // complex patterns
    const int Kp = 2 * K;              // realified columns
    const int rows = 1 << (nb - k);    // tile columns = GEMM rows
    const int nblk = rows >> 7;        // 128-row blocks
    const size_t half = (size_t)rows * Kp;   // floats per operand part
    float *ahi = aop, *alo = aop + half;
    const float *bhi = bop, *blo = bop + (size_t)Kp * Kp;
    // stage the tile as A = X^T (row o: Re x then Im x), tf32 hi and lo
    for (int o = threadIdx.x; o < rows; o += blockDim.x) {
        const uint32_t base = dense_row_base((uint32_t)o, gmask, nb);
        const int blk = o >> 7, m = o & 127;
        const size_t boff = (size_t)blk * 128 * Kp * 4;
        for (int r4 = 0; r4 < K; r4 += 4) {
            float re[4], im[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float2 v = tile[swz<float>((int)(base | (uint32_t)dep[r4 + i]), swm)];
                re[i] = v.x;
                im[i] = v.y;
            }
            float4 h, l;
            h = make_float4(to_tf32(re[0]), to_tf32(re[1]), to_tf32(re[2]), to_tf32(re[3]));
            l = make_float4(to_tf32(re[0] - h.x), to_tf32(re[1] - h.y), to_tf32(re[2] - h.z), to_tf32(re[3] - h.w));
            const uint32_t ore = dense_k_operand_offset((uint32_t)m, (uint32_t)r4, (uint32_t)Kp);
            *reinterpret_cast<float4 *>(reinterpret_cast<char *>(ahi) + boff + ore) = h;
            *reinterpret_cast<float4 *>(reinterpret_cast<char *>(alo) + boff + ore) = l;
            h = make_float4(to_tf32(im[0]), to_tf32(im[1]), to_tf32(im[2]), to_tf32(im[3]));
            l = make_float4(to_tf32(im[0] - h.x), to_tf32(im[1] - h.y), to_tf32(im[2] - h.z), to_tf32(im[3] - h.w));
            const uint32_t oim = dense_k_operand_offset((uint32_t)m, (uint32_t)(K + r4), (uint32_t)Kp);
            *reinterpret_cast<float4 *>(reinterpret_cast<char *>(ahi) + boff + oim) = h;
            *reinterpret_cast<float4 *>(reinterpret_cast<char *>(alo) + boff + oim) = l;
        }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        tmem_fence_after();
        const uint32_t idesc = umma_tf32_idesc(128, Kp);
        const uint32_t sa_hi = smem_u32(ahi), sa_lo = smem_u32(alo), sb_hi = smem_u32(bhi), sb_lo = smem_u32(blo);
        for (int b = 0; b < nblk; ++b) {
            const uint32_t d = d_tmem + (uint32_t)(b * Kp);
            const uint32_t boff = (uint32_t)b * 128u * (uint32_t)Kp * 4u;
            for (int st = 0; st < Kp / 8; ++st) {
                const uint32_t so = (uint32_t)st * 256u;   // 8 columns = two 4-column core matrices
                const uint64_t ah = umma_kmajor_desc(sa_hi + boff + so, (uint32_t)Kp);
                const uint64_t al = umma_kmajor_desc(sa_lo + boff + so, (uint32_t)Kp);
                const uint64_t bh = umma_kmajor_desc(sb_hi + so, (uint32_t)Kp);
                const uint64_t bl = umma_kmajor_desc(sb_lo + so, (uint32_t)Kp);
                umma_tf32(d, ah, bh, idesc, st > 0 ? 1u : 0u);
                umma_tf32(d, ah, bl, idesc, 1u);
                umma_tf32(d, al, bh, idesc, 1u);
            }
        }
        umma_commit(bar);
    }
    const bool mine = mbar_wait_bounded(bar, parity);
    const bool ok = __syncthreads_and(mine) != 0;
    if (!ok) return false;
    tmem_fence_after();
    // read back: warp w reads TMEM lanes 32 (w % 4) .. of blocks w / 4, w / 4 + 2, ...
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    for (int b = warp >> 2; b < nblk; b += nwarps >> 2) {
        const int o = b * 128 + 32 * (warp & 3) + lane;
        const uint32_t base = dense_row_base((uint32_t)o, gmask, nb);
        const uint32_t taddr = d_tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(b * Kp);
        for (int c0 = 0; c0 < K; c0 += 16) {
            // Re y[c0 .. c0+15] at columns c0.., Im at K + c0 ..
            float re[16], im[16];
            tmem_ld16(taddr + (uint32_t)c0, re);
            tmem_ld16(taddr + (uint32_t)(K + c0), im);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (c0 + i < K) tile[swz<float>((int)(base | (uint32_t)dep[c0 + i]), swm)] = make_float2(re[i], im[i]);
        }
    }
    tmem_fence_before();
    __syncthreads();
    return true;
}

// complex128: y = G x per tile column on the CUDA cores (G in shared memory).
__device__ void tile_dense_k_f64(double2 *tile, int nb, int swm, int k, const int32_t *dep, uint32_t gmask,
                                 const double2 *g) {
    const int K = 1 << k;
    const int rows = 1 << (nb - k);
    for (int o = threadIdx.x; o < rows; o += blockDim.x) {
        const uint32_t base = dense_row_base((uint32_t)o, gmask, nb);
        double2 x[1 << kMaxDenseK];
#pragma unroll
        for (int c = 0; c < (1 << kMaxDenseK); ++c)
            if (c < K) x[c] = tile[swz<double>((int)(base | (uint32_t)dep[c]), swm)];
        for (int r = 0; r < K; ++r) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < (1 << kMaxDenseK); ++c)
                if (c < K) acc = cfma(g[r * K + c], x[c], acc);
            tile[swz<double>((int)(base | (uint32_t)dep[r]), swm)] = acc;
        }
    }
    __syncthreads();
}

// kDense: the pass applies the dense k-qubit gate a.dense over every tile
// (tile_dense_k_tc / tile_dense_k_f64) instead of the register sweeps.
// kC, kJ: compile-time chunk log2 and tile qubits (0: from the args).
template <typename R, bool kCodes, bool kDense, int kC, int kJ>
__global__ void __launch_bounds__(kStagedThreads, 1) staged_pass_kernel(const PassArgs a) {
    using T = typename Cplx<R>::T;
    extern __shared__ __align__(128) unsigned char staged_smem[];
    unsigned char *smem = staged_smem;
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ __align__(8) uint64_t s_mma;   // dense complex64: MMA completion
    __shared__ uint32_t s_tmem;               // dense complex64: TMEM base address
    __shared__ unsigned long long s_tile_off, s_next, s_slab_end;
    __shared__ int s_flag;
    __shared__ int32_t s_tq[kMaxTileQubits];
    __shared__ int8_t s_oq[kMaxOuterSel];

    const int C = kC ? kC : a.C, j = kJ ? kJ : a.j, nb = C + j;
    const int nchunks = 1 << j;
    const int ncomp = 2 << C;
    const int per_lane = ncomp >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int blk_shift = a.B - C;
    const int swm = swizzle_mask<R>(C);
    const uint32_t nblk = 1u << (a.n - a.B);
    const bool smask = nblk <= kMaxSmemBlocks;
    const uint32_t mask_words = smask ? (nblk + 31) / 32 : 0;
    const StagedLayout Ly = staged_layout(sizeof(R) == 8, C, j, mask_words, kDense ? a.dense.k : 0);

    T *tile = reinterpret_cast<T *>(smem + Ly.tile);
    // the two slots of each double-buffered region, by pointer arithmetic
    // (no arrays indexed at run time, which would live in local memory)
    auto buf = [&](int s) { return reinterpret_cast<uint32_t *>(smem + Ly.buf0 + (size_t)s * (Ly.buf1 - Ly.buf0)); };
    auto hdr = [&](int s) { return reinterpret_cast<ChunkMeta *>(smem + Ly.hdr0 + (size_t)s * (Ly.hdr1 - Ly.hdr0)); };
    auto poff = [&](int s) { return reinterpret_cast<uint32_t *>(smem + Ly.poff0 + (size_t)s * (Ly.poff1 - Ly.poff0)); };
    int32_t *s_base = reinterpret_cast<int32_t *>(smem + Ly.base);
    uint32_t *s_width = reinterpret_cast<uint32_t *>(smem + Ly.width);
    uint32_t *s_nz = reinterpret_cast<uint32_t *>(smem + Ly.nz);
    unsigned long long *s_off = reinterpret_cast<unsigned long long *>(smem + Ly.off);
    uint32_t *s_act = reinterpret_cast<uint32_t *>(smem + Ly.act);
    uint32_t *s_sto = reinterpret_cast<uint32_t *>(smem + Ly.sto);

    if (threadIdx.x < kMaxTileQubits) s_tq[threadIdx.x] = a.tq[threadIdx.x];
    if (threadIdx.x < kMaxOuterSel) s_oq[threadIdx.x] = a.outer_q[threadIdx.x];
    if (threadIdx.x == 0) {
        s_next = 0;
        s_slab_end = 0;
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // block bitmasks: bit b of s_act = block b's group is active this stage,
    // of s_sto = block b was stored when the stage began
    for (uint32_t b0 = (uint32_t)warp * 32; b0 < mask_words * 32; b0 += (uint32_t)nwarps * 32) {
        const uint32_t b = b0 + lane;
        const bool act = b < nblk && a.group_active[a.block_to_group[b]] != 0;
        const bool sto = b < nblk && a.mask[b] != 0;
        const uint32_t wa = __ballot_sync(0xffffffffu, act), ws = __ballot_sync(0xffffffffu, sto);
        if (lane == 0) {
            s_act[b0 >> 5] = wa;
            s_sto[b0 >> 5] = ws;
        }
    }
    // dense gate: its pattern offsets and matrix operands into shared memory;
    // complex64 also allocates the TMEM accumulator (warp 0)
    int32_t *dense_dep = nullptr;
    uint32_t dense_gmask = 0, mma_phase = 0;
    bool mma_stuck = false;      // a bounded MMA wait gave up: wait again before freeing TMEM
    if constexpr (kDense) {
        const int K = 1 << a.dense.k;
        dense_dep = reinterpret_cast<int32_t *>(smem + Ly.dense_dep);
        for (int r = threadIdx.x; r < K; r += blockDim.x) {
            int32_t d = 0;
            for (int i = 0; i < a.dense.k; ++i) d |= ((r >> i) & 1) << a.dense.pos[i];
            dense_dep[r] = d;
        }
        for (int i = 0; i < a.dense.k; ++i) dense_gmask |= 1u << a.dense.pos[i];
        if constexpr (sizeof(R) == 4) {
            const size_t nf = (size_t)4 << (2 * a.dense.k);  // floats per operand part
            float *bop = reinterpret_cast<float *>(smem + Ly.dense_b);
            for (size_t i = threadIdx.x; i < nf; i += blockDim.x) {
                bop[i] = a.dense.bhi[i];
                bop[nf + i] = a.dense.blo[i];
            }
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            if (threadIdx.x == 0) {
                mbar_init(&s_mma, 1);
                asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
            }
            if (warp == 0) {
                asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                                 smem_u32(&s_tmem)),
                             "r"(kDenseTmemCols)
                             : "memory");
                asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
            }
            tmem_fence_before();
        } else {
            const size_t nm = (size_t)2 << (2 * a.dense.k);  // doubles
            double *g = reinterpret_cast<double *>(smem + Ly.dense_b);
            for (size_t i = threadIdx.x; i < nm; i += blockDim.x) g[i] = a.dense.mat[i];
        }
    }
    __syncthreads();
    if constexpr (kDense && sizeof(R) == 4) tmem_fence_after();

    auto block_active = [&](uint64_t blk) -> bool {
        return smask ? ((s_act[blk >> 5] >> (blk & 31)) & 1u) != 0 : a.group_active[a.block_to_group[blk]] != 0;
    };
    auto block_stored = [&](uint64_t blk) -> bool {
        return smask ? ((s_sto[blk >> 5] >> (blk & 31)) & 1u) != 0 : a.mask[blk] != 0;
    };
    // this CTA's first tile at or after t (t in its sequence) whose group is
    // active; ~0 when none is left (uniform across the CTA)
    auto next_active = [&](uint64_t t) -> uint64_t {
        for (; t < a.n_tiles; t += gridDim.x)
            if (block_active(insert_zero_bits(t, s_tq, j) >> blk_shift)) return t;
        return ~0ull;
    };
    // headers of tile t into hdr(s) (16-byte cp.async copies; a chunk of a
    // block that is not stored at the start of the stage reads as zeros on
    // the stage's first pass and its header is not read)
    auto load_headers = [&](uint64_t t, int s) {
        const uint64_t cb = insert_zero_bits(t, s_tq, j);
        for (int c = threadIdx.x; c < nchunks; c += blockDim.x) {
            const uint64_t chunk = cb | deposit_bits((uint32_t)c, s_tq, j);
            if (!a.first_pass || block_stored(chunk >> blk_shift)) cp_async16(&hdr(s)[c], &a.meta_in[chunk]);
            else hdr(s)[c] = ChunkMeta{0, 0, 0};
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    // warp 0: payload copies of the tile whose headers are in hdr(s) into
    // buf(s); chunk c's payload lands at byte poff(s)[c]
    auto issue_payload = [&](int s) {
        uint32_t run = 0;
        for (int c0 = 0; c0 < nchunks; c0 += 32) {
            const int c = c0 + lane;
            const uint32_t w = c < nchunks ? hdr(s)[c].width : 0u;
            const uint32_t sz = (uint32_t)payload_bytes(C, w > 32 ? 32u : w);
            uint32_t incl = sz;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t2 = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t2;
            }
            if (c < nchunks) poff(s)[c] = run + incl - sz;
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        // the buffer was last read by generic loads (the decode of two tiles ago)
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        if (lane == 0) mbar_arrive_expect_tx(&s_bar[s], run);
        __syncwarp();
        for (int c = lane; c < nchunks; c += 32) {
            const ChunkMeta md = hdr(s)[c];
            const uint32_t sz = (uint32_t)payload_bytes(C, md.width > 32 ? 32u : md.width);
            if (sz) bulk_copy_g2s(reinterpret_cast<unsigned char *>(buf(s)) + poff(s)[c],
                                  reinterpret_cast<const unsigned char *>(a.arena_in) + md.offset, sz, &s_bar[s]);
        }
    };

    unsigned long long rd = 0, wr = 0, ntiles = 0;
    uint32_t phase = 0u;    // bit s: parity of the next phase of s_bar[s]
    uint32_t pending = 0u;  // bit s: a payload fill of buf(s) not yet waited for

    uint64_t cur = next_active(blockIdx.x);
    uint64_t nxt = cur == ~0ull ? ~0ull : next_active(cur + gridDim.x);
    if (cur != ~0ull) {
        load_headers(cur, 0);
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        if (warp == 0) issue_payload(0);
        pending |= 1u;
        if (nxt != ~0ull) load_headers(nxt, 1);
    }

    for (int it = 0; cur != ~0ull; ++it) {
        const int slot = it & 1;
        const uint64_t chunk_base = insert_zero_bits(cur, s_tq, j);
        // error flag of this tile, tested at its reservation
        int err_seen = 0;
        if (threadIdx.x == 0) err_seen = *reinterpret_cast<volatile int32_t *>(a.error);
        // headers of the next tile (issued one tile ago) and this tile's payload
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        const bool mine = mbar_wait_bounded(&s_bar[slot], (phase >> slot) & 1u);
        const bool ok = __syncthreads_and(mine) != 0;  // uniform: every thread saw the fill complete
        if (!ok) {
            if (threadIdx.x == 0) atomicExch(a.error, 2);
            break;
        }
        phase ^= 1u << slot;
        pending &= ~(1u << slot);
        ++ntiles;
        const uint64_t nxt2 = nxt == ~0ull ? ~0ull : next_active(nxt + gridDim.x);
        if (nxt != ~0ull) {
            if (warp == 0) issue_payload(slot ^ 1);
            pending |= 1u << (slot ^ 1);
        }

        // ---- decode this tile's chunks from buf(slot) into the value tile
        for (int c = warp; c < nchunks; c += nwarps) {
            const ChunkMeta md = hdr(slot)[c];
            unpack_chunk<R, TileSlot<R>, kCodes>(md, per_lane, a.codec, reinterpret_cast<R *>(tile),
                                                 buf(slot) + (poff(slot)[c] >> 2), lane, TileSlot<R>{c << C, swm});
            if (lane == 0) {
                const uint64_t chunk = chunk_base | deposit_bits((uint32_t)c, s_tq, j);
                if (!a.first_pass || block_stored(chunk >> blk_shift))
                    rd += payload_bytes(C, md.width) + sizeof(ChunkMeta);
            }
        }
        __syncthreads();
        // hdr(slot) is free: the headers of the tile after the next one
        if (nxt2 != ~0ull) load_headers(nxt2, slot);

        // ---- gates
        if constexpr (kDense) {
            if constexpr (sizeof(R) == 4) {
                const bool done = tile_dense_k_tc(reinterpret_cast<float2 *>(tile), nb, swm, a.dense.k, dense_dep,
                                                  dense_gmask, reinterpret_cast<float *>(smem + Ly.dense_a),
                                                  reinterpret_cast<const float *>(smem + Ly.dense_b), s_tmem,
                                                  &s_mma, mma_phase);
                if (!done) {
                    mma_stuck = true;
                    if (threadIdx.x == 0) atomicExch(a.error, 2);
                    break;
                }
                mma_phase ^= 1u;
            } else {
                tile_dense_k_f64(reinterpret_cast<double2 *>(tile), nb, swm, a.dense.k, dense_dep, dense_gmask,
                                 reinterpret_cast<const double2 *>(smem + Ly.dense_b));
            }
        } else {
            tile_sweeps<R, kRegBits>(tile, nb, swm, a.sweeps, a.nsweeps, a.ops, reinterpret_cast<const T *>(a.pool),
                                     outer_word(chunk_base << C, s_oq, a.nouter));
            if constexpr (!kCodes) {
                // buf(slot) is free here: it holds the tile's term coefficients
                if (a.diag.nterms)
                    tile_diag_sum<R>(tile, nb, swm, a.diag, chunk_base << C, reinterpret_cast<double *>(buf(slot)));
            }
        }

        // ---- quantise (codes replace values in shared memory)
        for (int c = warp; c < nchunks; c += nwarps) {
            R *comp = reinterpret_cast<R *>(tile) + (size_t)c * ncomp;
            int32_t base;
            uint32_t width;
            bool nz;
            quantize_chunk<R, TileSlot<R>, kCodes>(reinterpret_cast<R *>(tile), per_lane, a.codec, a.exact_zero != 0,
                                                   lane, &base, &width, &nz, TileSlot<R>{c << C, swm},
                                                   reinterpret_cast<int32_t *>(comp));
            if (lane == 0) {
                s_base[c] = base;
                s_width[c] = width;
                s_nz[c] = nz ? 1u : 0u;
            }
        }
        __syncthreads();

        // ---- reserve the tile's output bytes (warp 0 scans the chunk sizes)
        if (warp == 0) {
            const int per = (nchunks + 31) >> 5;
            const int c0 = lane * per;
            unsigned long long mine = 0;
            for (int c = c0; c < c0 + per && c < nchunks; ++c) mine += payload_bytes(C, s_width[c]);
            unsigned long long incl = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long t2 = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t2;
            }
            unsigned long long run = incl - mine;
            for (int c = c0; c < c0 + per && c < nchunks; ++c) {
                s_off[c] = run;
                run += payload_bytes(C, s_width[c]);
            }
            const unsigned long long total = __shfl_sync(0xffffffffu, incl, 31);
            if (lane == 0) {
                unsigned long long off = s_next;
                s_flag = err_seen;
                if (!err_seen && (a.slab == 0 || off + total > s_slab_end)) {
                    const unsigned long long want = total > a.slab ? total : a.slab;
                    off = atomicAdd(a.bump, want);
                    if (off + want > a.capacity) {
                        atomicExch(a.error, 1);
                        s_flag = 1;
                    }
                    s_slab_end = off + want;
                }
                s_tile_off = off;
                s_next = off + total;
                if (!s_flag) wr += total + (unsigned long long)nchunks * sizeof(ChunkMeta);
            }
        }
        __syncthreads();
        if (s_flag) break;

        // ---- pack and store
        for (int c = warp; c < nchunks; c += nwarps) {
            const uint64_t chunk = apply_perm(a.perm, chunk_base | deposit_bits((uint32_t)c, s_tq, j));
            const int32_t *codes = reinterpret_cast<const int32_t *>(reinterpret_cast<R *>(tile) + (size_t)c * ncomp);
            const unsigned long long off = s_tile_off + s_off[c];
            const uint32_t w = s_width[c];
            pack_chunk(codes, per_lane, s_base[c], w, a.arena_out + (off >> 2), lane);
            if (lane == 0) {
                ChunkMeta md;
                md.offset = off;
                md.base = s_base[c];
                md.width = w;
                a.meta_out[chunk] = md;
                if (a.final_pass) {
                    const uint64_t blk = chunk >> blk_shift;
                    if (s_nz[c]) atomicOr(&a.block_nz[blk], 1u);
                    atomicAdd(&a.block_bytes[blk], (unsigned long long)(payload_bytes(C, w) + sizeof(ChunkMeta)));
                }
            }
        }
        cur = nxt;
        nxt = nxt2;
    }
    // a CTA that stopped early still has copies in flight into its shared
    // memory: wait for them (bounded) before it exits
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    for (int s = 0; s < 2; ++s)
        if ((pending >> s) & 1u) (void)mbar_wait_bounded(&s_bar[s], (phase >> s) & 1u);
    __syncthreads();
    if constexpr (kDense && sizeof(R) == 4) {
        // every MMA was waited for (or its bounded wait gave up and the loop
        // stopped); the accumulator is freed by the warp that allocated it
        if (mma_stuck) (void)mbar_wait_bounded(&s_mma, mma_phase);
        tmem_fence_after();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(s_tmem),
                         "r"(kDenseTmemCols)
                         : "memory");
    }
    if (rd) atomicAdd(&a.stats[0], rd);
    if (threadIdx.x == 0) {
        if (wr) atomicAdd(&a.stats[1], wr);
        if (ntiles) atomicAdd(&a.stats[2], ntiles);
    }
}

// ------------------------------------------------------------ header permutation pass
__global__ void perm_pass_kernel(const PermPassArgs a) {
    const int blk_shift = a.B - a.C;
    const int lane = threadIdx.x & 31;
    const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long moved = 0;
    // every lane of a warp runs the same iterations, so the per-block sums
    // below can use warp-wide match and reduce
    for (uint64_t c0 = warp0 * 32; c0 < a.nchunks; c0 += nwarps * 32) {
        const uint64_t c = c0 + lane;
        bool live = c < a.nchunks;
        const uint64_t blk = c >> blk_shift;
        if (live) live = a.group_active[a.block_to_group[blk]] != 0;
        uint64_t ob = ~0ull;
        uint32_t bytes = 0, nz = 0;
        if (live) {
            ChunkMeta md{0, 0, 0};
            if (!a.first_pass || a.mask[blk]) md = a.meta_in[c];
            const uint64_t oc = apply_perm(a.perm, c);
            a.meta_out[oc] = md;
            ++moved;
            ob = oc >> blk_shift;
            bytes = (uint32_t)(payload_bytes(a.C, md.width) + sizeof(ChunkMeta));
            nz = (md.width != 0 || md.base != 0) ? 1u : 0u;
        }
        if (a.final_pass) {
            const unsigned grp = __match_any_sync(0xffffffffu, ob);
            const uint32_t gbytes = __reduce_add_sync(grp, bytes);
            const uint32_t gnz = __reduce_or_sync(grp, nz);
            if (live && lane == __ffs(grp) - 1) {
                if (gnz) atomicOr(&a.block_nz[ob], 1u);
                atomicAdd(&a.block_bytes[ob], (unsigned long long)gbytes);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(0xffffffffu, moved, o);
    if (lane == 0 && moved) {
        atomicAdd(&a.stats[0], moved * sizeof(ChunkMeta));
        atomicAdd(&a.stats[1], moved * sizeof(ChunkMeta));
    }
}

// ------------------------------------------------------------ dense pass
// kC, kJ: the chunk and tile-qubit counts as compile-time constants (0 = read
// them from the launch arguments).
template <typename R, int RB, int kC, int kJ>
__global__ void __launch_bounds__(kSweepThreads, 3) dense_pass_kernel(const DensePassArgs a) {
    using T = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    T *tile = reinterpret_cast<T *>(smem);
    T *st = reinterpret_cast<T *>(a.state);
    const int C = kC ? kC : a.C, j = kJ ? kJ : a.j, nb = C + j;
    const int size = 1 << nb;
    const int cmask = (1 << C) - 1;
    const int swm = swizzle_mask<R>(C);
    __shared__ int32_t s_tq[kMaxTileQubits];
    __shared__ int8_t s_oq[kMaxOuterSel];
    if (threadIdx.x < kMaxTileQubits) s_tq[threadIdx.x] = a.tq[threadIdx.x];
    if (threadIdx.x < kMaxOuterSel) s_oq[threadIdx.x] = a.outer_q[threadIdx.x];
    __syncthreads();
    for (uint64_t tile_id = blockIdx.x; tile_id < a.n_tiles; tile_id += gridDim.x) {
        const uint64_t chunk_base = insert_zero_bits(tile_id, s_tq, j);
        for (int e = threadIdx.x; e < size; e += blockDim.x) {
            const uint64_t amp = ((chunk_base | deposit_bits((uint32_t)(e >> C), s_tq, j)) << C) | (uint64_t)(e & cmask);
            tile[swz<R>(e, swm)] = st[amp];
        }
        __syncthreads();
        tile_sweeps<R, RB>(tile, nb, swm, a.sweeps, a.nsweeps, a.ops, reinterpret_cast<const T *>(a.pool),
                           outer_word(chunk_base << C, s_oq, a.nouter));
        for (int e = threadIdx.x; e < size; e += blockDim.x) {
            const uint64_t amp = ((chunk_base | deposit_bits((uint32_t)(e >> C), s_tq, j)) << C) | (uint64_t)(e & cmask);
            st[amp] = tile[swz<R>(e, swm)];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ plain per-gate
template <typename R>
__global__ void pergate_kernel(typename Cplx<R>::T *st, int n, const KGate *__restrict__ gp) {
    using T = typename Cplx<R>::T;
    const KGate &g = *gp;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    if (g.nq == 1) {
        const int p = g.q[0];
        const T e0 = make_c<T, R>(g.m[0], g.m[1]), e1 = make_c<T, R>(g.m[2], g.m[3]);
        const T e2 = make_c<T, R>(g.m[4], g.m[5]), e3 = make_c<T, R>(g.m[6], g.m[7]);
        const uint64_t half = uint64_t(1) << (n - 1), low = (uint64_t(1) << p) - 1;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half; i += stride) {
            const uint64_t i0 = ((i & ~low) << 1) | (i & low), i1 = i0 | (uint64_t(1) << p);
            const T a = st[i0], b = st[i1];
            st[i0] = cfma(e0, a, cmul(e1, b));
            st[i1] = cfma(e2, a, cmul(e3, b));
        }
    } else {
        const int pa = g.q[0], pb = g.q[1];
        T m[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) m[k] = make_c<T, R>(g.m[2 * k], g.m[2 * k + 1]);
        const uint64_t quarter = uint64_t(1) << (n - 2);
        const uint64_t mlo = (uint64_t(1) << pa) - 1, mhi = (uint64_t(1) << pb) - 1;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < quarter; i += stride) {
            uint64_t b = ((i & ~mlo) << 1) | (i & mlo);
            b = ((b & ~mhi) << 1) | (b & mhi);
            const uint64_t ia = uint64_t(1) << pa, ib = uint64_t(1) << pb;
            const T v0 = st[b], v1 = st[b | ia], v2 = st[b | ib], v3 = st[b | ia | ib];
            T o[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                T acc = cmul(m[4 * r], v0);
                acc = cfma(m[4 * r + 1], v1, acc);
                acc = cfma(m[4 * r + 2], v2, acc);
                acc = cfma(m[4 * r + 3], v3, acc);
                o[r] = acc;
            }
            st[b] = o[0];
            st[b | ia] = o[1];
            st[b | ib] = o[2];
            st[b | ia | ib] = o[3];
        }
    }
}

// ------------------------------------------------------------ stage bookkeeping
__global__ void stage_clear_kernel(uint8_t *group_active, uint32_t num_groups, uint32_t *block_nz,
                                   unsigned long long *block_bytes, uint32_t nb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < num_groups) group_active[i] = 0;
    if (i < nb) {
        block_nz[i] = 0;
        block_bytes[i] = 0;
    }
}

__global__ void stage_mark_kernel(const uint32_t *block_to_group, const uint8_t *mask, uint32_t nb,
                                  uint8_t *group_active) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb && mask[b]) group_active[block_to_group[b]] = 1;
}

// Blocks of active groups (all of them are processed, Q8): the stage's
// amplitude count is this times 2^B.
__global__ void stage_count_kernel(const uint32_t *block_to_group, const uint8_t *group_active, uint32_t nb,
                                   unsigned long long *count) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = (b < nb && group_active[block_to_group[b]]) ? 1ull : 0ull;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(count, v);
}

// Zero-mask rule of the reference (compressed_state.hpp:1015-1026,
// compressed_state_cuda.cu:282-305): only blocks that were zero before the
// stage and belong to an active group are tested; a stored block stays
// stored.
__global__ void stage_end_kernel(const uint32_t *block_to_group, const uint8_t *group_active, uint32_t nb,
                                 const uint32_t *block_nz, const unsigned long long *acc, uint8_t *mask,
                                 unsigned long long *block_bytes, unsigned long long *history_slot) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long bytes = 0;
    if (b < nb) {
        uint8_t mk = mask[b];
        if (group_active[block_to_group[b]]) {
            if (!mk && block_nz[b]) mk = 1;
            mask[b] = mk;
            bytes = mk ? acc[b] : 0ull;
        } else {
            bytes = mk ? block_bytes[b] : 0ull;
        }
        block_bytes[b] = bytes;
    }
    for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if ((threadIdx.x & 31) == 0 && bytes) atomicAdd(history_slot, bytes);
}

// Clears *out when some block of the mask is not stored (the caller sets it
// to 1 first); at most one store per CTA.  out may be the device alias of
// mapped host memory, which the host reads once the stream has passed this
// kernel: no copy-engine transfer, so the read does not queue behind
// another stream's large copies.
__global__ void mask_full_kernel(const uint8_t *mask, uint32_t nb, uint32_t *out) {
    int all = 1;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        all &= mask[b] != 0;
    all = __syncthreads_and(all);
    if (threadIdx.x == 0 && !all) *reinterpret_cast<volatile uint32_t *>(out) = 0u;
}

// Copies up to four device word arrays into dst (back to back), the device
// alias of mapped host memory: the end-of-apply counters reach the host
// without a copy-engine transfer.
__global__ void readback_kernel(ReadbackList l, unsigned long long *dst) {
    size_t o = 0;
    for (int k = 0; k < l.n; ++k) {
        for (size_t i = threadIdx.x; i < l.words[k]; i += blockDim.x) dst[o + i] = l.src[k][i];
        o += l.words[k];
    }
}

__global__ void sum_mask_bytes_kernel(const uint8_t *mask, const unsigned long long *bb, uint32_t nb,
                                      unsigned long long *out) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long v = (b < nb && mask[b]) ? bb[b] : 0ull;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(out, v);
}

// ------------------------------------------------------------ readout / norm
template <typename R>
__global__ void readout_kernel(const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B, int C,
                               CodecParams p, uint64_t chunk0, uint64_t nchunks, double *out, double scale) {
    __shared__ __align__(16) uint32_t stage[kPassThreads / 32][kStageWords];
    __shared__ R vals[kPassThreads / 32][2 << kMaxChunkLog2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ncomp = 2 << C, per_lane = ncomp >> 5;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = gw; k < nchunks; k += nw) {
        const uint64_t chunk = chunk0 + k;
        double *o = out + k * (uint64_t)ncomp;
        if (!mask[chunk >> (B - C)]) {
            for (int i = 0; i < per_lane; ++i) o[lane + 32 * i] = 0.0;
            continue;
        }
        decode_chunk<R>(arena, meta[chunk], per_lane, p, vals[warp], stage[warp], lane);
        for (int i = 0; i < per_lane; ++i) o[lane + 32 * i] = (double)vals[warp][lane + 32 * i] * scale;
        __syncwarp();
    }
}

// ------------------------------------------------------------ sampling
// |a|^2 of amplitude a of a decoded chunk as x*x + y*y, rounded after each
// operation (no fused multiply-add), so that the sums below are the ones of
// the reference's std::norm loop (compressed_state.hpp:1615-1616).
template <typename R>
__device__ __forceinline__ double amp_norm(const R *vals, int a) {
    const double x = (double)vals[2 * a], y = (double)vals[2 * a + 1];
    return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

// Sequential FP64 mass of every block, one warp per block: the warp decodes
// the block's chunks in order and lane 0 adds |a|^2 amplitude by amplitude,
// the reference's order (compressed_state.hpp:1613-1619), so block_mass is
// bit-identical to its `mass` for the same decoded amplitudes.  prefix[k] is
// the running sum when chunk k of the block begins, so that the cumulative
// distribution inside any chunk can be rebuilt exactly.  Zero blocks get 0.
template <typename R>
__global__ void block_mass_kernel(const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B, int C,
                                  CodecParams p, uint32_t nblocks, double *prefix, double *block_mass) {
    __shared__ __align__(16) uint32_t stage[kPassThreads / 32][kStageWords];
    __shared__ R vals[kPassThreads / 32][2 << kMaxChunkLog2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int namps = 1 << C, per_lane = (2 << C) >> 5;
    const uint32_t cpb = 1u << (B - C);
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t b = gw; b < nblocks; b += nw) {
        const uint64_t k0 = b * cpb;
        if (!mask[b]) {
            for (uint32_t k = lane; k < cpb; k += 32) prefix[k0 + k] = 0.0;
            if (lane == 0) block_mass[b] = 0.0;
            continue;
        }
        double acc = 0.0;
        for (uint32_t k = 0; k < cpb; ++k) {
            decode_chunk<R>(arena, meta[k0 + k], per_lane, p, vals[warp], stage[warp], lane);
            __syncwarp();
            if (lane == 0) {
                prefix[k0 + k] = acc;
                for (int a = 0; a < namps; ++a) acc = __dadd_rn(acc, amp_norm(vals[warp], a));
            }
            __syncwarp();
        }
        if (lane == 0) block_mass[b] = acc;
    }
}

// One shot per warp: the first amplitude j of block shot_block[s] whose
// sequential cumulative |a|^2 reaches rin[s] (std::lower_bound over the
// block's cdf, compressed_state.hpp:1652-1662), clamped to the block's last
// amplitude.  The chunk is found by a binary search over the chunk-end sums
// (prefix of the next chunk, block_mass for the last); inside it the running
// sum restarts from prefix[chunk] and repeats the same additions.  A zero
// block has an all-zero cdf, so its answer is j = 0.  out[s] = b * 2^B + j.
template <typename R>
__global__ void sample_in_block_kernel(const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B,
                                       int C, CodecParams p, const double *prefix, const double *block_mass,
                                       const uint32_t *shot_block, const double *rin, uint64_t nshots,
                                       uint64_t *out) {
    __shared__ __align__(16) uint32_t stage[kPassThreads / 32][kStageWords];
    __shared__ R vals[kPassThreads / 32][2 << kMaxChunkLog2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int namps = 1 << C, per_lane = (2 << C) >> 5;
    const uint32_t cpb = 1u << (B - C);
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t s = gw; s < nshots; s += nw) {
        const uint64_t b = shot_block[s];
        const uint64_t k0 = b * cpb;
        const double r = rin[s];
        if (!mask[b]) {
            if (lane == 0) out[s] = b << B;
            continue;
        }
        // first chunk whose end sum reaches r; the last chunk when none does
        uint32_t lo = 0, hi = cpb - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            const double end = prefix[k0 + mid + 1];
            if (end >= r) hi = mid;
            else lo = mid + 1;
        }
        const uint32_t k = lo;
        decode_chunk<R>(arena, meta[k0 + k], per_lane, p, vals[warp], stage[warp], lane);
        __syncwarp();
        if (lane == 0) {
            double acc = prefix[k0 + k];
            int j = namps - 1;
            for (int a = 0; a < namps; ++a) {
                acc = __dadd_rn(acc, amp_norm(vals[warp], a));
                if (acc >= r) {
                    j = a;
                    break;
                }
            }
            out[s] = (b << B) + ((uint64_t)k << C) + (uint64_t)j;
        }
        __syncwarp();
    }
}

template <typename R>
__global__ void norm_kernel(const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B, int C,
                            CodecParams p, uint64_t nchunks, double *out) {
    __shared__ __align__(16) uint32_t stage[kPassThreads / 32][kStageWords];
    __shared__ R vals[kPassThreads / 32][2 << kMaxChunkLog2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ncomp = 2 << C, per_lane = ncomp >> 5;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double acc = 0.0;
    for (uint64_t chunk = gw; chunk < nchunks; chunk += nw) {
        if (!mask[chunk >> (B - C)]) continue;
        decode_chunk<R>(arena, meta[chunk], per_lane, p, vals[warp], stage[warp], lane);
        for (int i = 0; i < per_lane; ++i) {
            const double v = (double)vals[warp][lane + 32 * i];
            acc = fma(v, v, acc);
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0 && acc != 0.0) atomicAdd(out, acc);
}

// Encode chunks from a device complex128 buffer into the store (load path).
template <typename R>
__global__ void encode_kernel(const double *vals, int B, int C, CodecParams p, uint64_t chunk0, uint64_t nchunks,
                              ChunkMeta *meta, uint32_t *arena, unsigned long long *bump, uint64_t capacity,
                              uint32_t *block_nz, unsigned long long *block_bytes, int32_t *error) {
    __shared__ R buf[kPassThreads / 32][2 << kMaxChunkLog2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ncomp = 2 << C, per_lane = ncomp >> 5;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = gw; k < nchunks; k += nw) {
        const uint64_t chunk = chunk0 + k;
        R *comp = buf[warp];
        for (int i = 0; i < per_lane; ++i) comp[lane + 32 * i] = (R)vals[k * (uint64_t)ncomp + lane + 32 * i];
        __syncwarp();
        int32_t base;
        uint32_t width;
        bool nz;
        quantize_chunk<R>(comp, per_lane, p, true, lane, &base, &width, &nz);
        const uint64_t bytes = payload_bytes(C, width);
        unsigned long long off = 0;
        if (lane == 0) off = atomicAdd(bump, (unsigned long long)bytes);
        off = __shfl_sync(0xffffffffu, off, 0);
        if (off + bytes > capacity) {
            if (lane == 0) atomicExch(error, 1);
            __syncwarp();
            continue;
        }
        pack_chunk(reinterpret_cast<const int32_t *>(comp), per_lane, base, width, arena + (off >> 2), lane);
        if (lane == 0) {
            ChunkMeta md;
            md.offset = off;
            md.base = base;
            md.width = width;
            meta[chunk] = md;
            const uint64_t blk = chunk >> (B - C);
            if (nz) atomicOr(&block_nz[blk], 1u);
            atomicAdd(&block_bytes[blk], (unsigned long long)(bytes + sizeof(ChunkMeta)));
        }
        __syncwarp();
    }
}

template <typename R>
__global__ void codec_test_kernel(const R *vals, int C, CodecParams p, uint64_t nchunks, uint32_t *words,
                                  int32_t *bases, uint32_t *widths, R *decoded) {
    __shared__ __align__(16) uint32_t stage[kPassThreads / 32][kStageWords];
    __shared__ R buf[kPassThreads / 32][2 << kMaxChunkLog2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ncomp = 2 << C, per_lane = ncomp >> 5;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t max_words = (uint64_t)per_lane * 32;  // width 32
    for (uint64_t k = gw; k < nchunks; k += nw) {
        R *comp = buf[warp];
        for (int i = 0; i < per_lane; ++i) comp[lane + 32 * i] = vals[k * ncomp + lane + 32 * i];
        __syncwarp();
        int32_t base;
        uint32_t width;
        bool nz;
        quantize_chunk<R>(comp, per_lane, p, true, lane, &base, &width, &nz);
        uint32_t *dst = words + k * max_words;
        pack_chunk(reinterpret_cast<const int32_t *>(comp), per_lane, base, width, dst, lane);
        if (lane == 0) {
            bases[k] = base;
            widths[k] = width;
        }
        __syncwarp();
        __threadfence_block();
        ChunkMeta md;
        md.offset = 0;
        md.base = base;
        md.width = width;
        decode_chunk<R>(dst, md, per_lane, p, comp, stage[warp], lane);
        __syncwarp();
        for (int i = 0; i < per_lane; ++i) decoded[k * ncomp + lane + 32 * i] = comp[lane + 32 * i];
        __syncwarp();
    }
}

template <typename R>
__global__ void dense_norm_kernel(const R *s, uint64_t ncomp, double *out) {
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ncomp; i += (uint64_t)gridDim.x * blockDim.x) {
        const double v = (double)s[i];
        acc = fma(v, v, acc);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(out, acc);
}

template <typename R>
__global__ void to_c128_kernel(const R *s, uint64_t ncomp, double *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ncomp; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (double)s[i];
}

template <typename R>
__global__ void from_c128_kernel(const double *in, uint64_t ncomp, R *s) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ncomp; i += (uint64_t)gridDim.x * blockDim.x)
        s[i] = (R)in[i];
}

// ------------------------------------------------------------ Pauli expectation
constexpr int kExpectThreads = 256;
constexpr int kMaxTermsPerLaunch = 256;

__device__ __forceinline__ double block_warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename R>
__global__ void __launch_bounds__(kExpectThreads) expect_kernel(const ExpectArgs a) {
    using T = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_acc[2 * kMaxTermsPerLaunch];
    __shared__ int32_t s_tq[kMaxTileQubits];
    const int C = a.C, j = a.j, nb = C + j;
    const int nchunks = 1 << j;
    const int ncomp = 2 << C;
    const int per_lane = ncomp >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int blk_shift = a.B - C;
    const int swm = swizzle_mask<R>(C);
    const bool two = a.meta_bra != nullptr;
    T *tile = reinterpret_cast<T *>(smem);
    T *btile = two ? tile + ((size_t)1 << nb) : tile;  // bra tile (the ket tile itself without a bra store)
    uint32_t *wstage = reinterpret_cast<uint32_t *>(smem + ((two ? 2 * sizeof(T) : sizeof(T)) << nb)) + warp * kStageWords;
    for (int i = threadIdx.x; i < 2 * a.nterms; i += blockDim.x) s_acc[i] = 0.0;
    if (threadIdx.x < kMaxTileQubits) s_tq[threadIdx.x] = a.tq[threadIdx.x];
    __syncthreads();
    const int size = 1 << nb;
    for (uint64_t tile_id = blockIdx.x; tile_id < a.n_tiles; tile_id += gridDim.x) {
        const uint64_t chunk_base = insert_zero_bits(tile_id, s_tq, j);
        bool any = false, anyb = false;
        for (int c = 0; c < nchunks; ++c) {
            const uint64_t blk = (chunk_base | deposit_bits((uint32_t)c, s_tq, j)) >> blk_shift;
            any |= a.mask[blk] != 0;
            anyb |= two && a.mask_bra[blk] != 0;
        }
        if (!any || (two && !anyb)) continue;  // uniform: every thread reads the same mask bytes
        for (int side = 0; side < (two ? 2 : 1); ++side) {
            const ChunkMeta *meta = side ? a.meta_bra : a.meta;
            const uint32_t *arena = side ? a.arena_bra : a.arena;
            const uint8_t *mask = side ? a.mask_bra : a.mask;
            T *dst = side ? btile : tile;
            for (int c = warp; c < nchunks; c += nwarps) {
                const uint64_t chunk = chunk_base | deposit_bits((uint32_t)c, s_tq, j);
                R *comp = reinterpret_cast<R *>(dst) + (size_t)c * ncomp;
                if (!mask[chunk >> blk_shift]) {
                    for (int i = 0; i < per_lane; ++i) comp[lane + 32 * i] = R(0);
                    continue;
                }
                decode_chunk<R>(arena, meta[chunk], per_lane, a.codec, reinterpret_cast<R *>(dst), wstage, lane,
                                TileSlot<R>{c << C, swm});
            }
        }
        __syncthreads();
        const uint64_t base_amp = chunk_base << C;
        for (int t = 0; t < a.nterms; ++t) {
            const PauliTerm pt = a.terms[t];
            const int outer = __popcll(base_amp & pt.zo) & 1;
            double re = 0.0, im = 0.0;
            for (int x = threadIdx.x; x < size; x += blockDim.x) {
                const T ax = tile[swz<R>(x, swm)];
                const T by = btile[swz<R>(x ^ (int)pt.xt, swm)];
                // conj(by) * ax
                double pr = (double)by.x * (double)ax.x + (double)by.y * (double)ax.y;
                double pi = (double)by.x * (double)ax.y - (double)by.y * (double)ax.x;
                if ((__popc((uint32_t)x & pt.zt) + outer) & 1) { pr = -pr; pi = -pi; }
                re += pr;
                im += pi;
            }
            re = block_warp_sum(re);
            im = block_warp_sum(im);
            if (lane == 0) {
                atomicAdd(&s_acc[2 * t], re);
                atomicAdd(&s_acc[2 * t + 1], im);
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * a.nterms; i += blockDim.x)
        if (s_acc[i] != 0.0) atomicAdd(&a.out[i], s_acc[i]);
}

template <typename R>
__global__ void __launch_bounds__(kExpectThreads) dense_expect_kernel(const typename Cplx<R>::T *__restrict__ bra,
                                                                      const typename Cplx<R>::T *__restrict__ st, int n,
                                                                      const PauliTerm *terms, int nterms, double *out) {
    using T = typename Cplx<R>::T;
    __shared__ double s_acc[2 * kMaxTermsPerLaunch];
    const int lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < 2 * nterms; i += blockDim.x) s_acc[i] = 0.0;
    __syncthreads();
    const uint64_t dim = uint64_t(1) << n;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (int t = 0; t < nterms; ++t) {
        const PauliTerm pt = terms[t];
        double re = 0.0, im = 0.0;
        for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += stride) {
            const T ax = st[x];
            const T by = bra[x ^ pt.xg];
            double pr = (double)by.x * (double)ax.x + (double)by.y * (double)ax.y;
            double pi = (double)by.x * (double)ax.y - (double)by.y * (double)ax.x;
            if (__popcll(x & pt.zg) & 1) { pr = -pr; pi = -pi; }
            re += pr;
            im += pi;
        }
        re = block_warp_sum(re);
        im = block_warp_sum(im);
        if (lane == 0) {
            atomicAdd(&s_acc[2 * t], re);
            atomicAdd(&s_acc[2 * t + 1], im);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * nterms; i += blockDim.x)
        if (s_acc[i] != 0.0) atomicAdd(&out[i], s_acc[i]);
}

// ------------------------------------------------------------ adjoint backward pass
// One gate on a shared-memory tile (linear layout); the gate's qubits outside
// the tile are fixed by base_amp and must be non-mixing.
template <typename R>
__device__ void smem_apply_gate(typename Cplx<R>::T *t, int nb, const KGate &g, uint64_t base_amp) {
    using T = typename Cplx<R>::T;
    const int dim = 1 << g.nq;
    int pos[2] = {-1, -1}, fixv[2] = {0, 0};
    for (int i = 0; i < g.nq; ++i) {
        pos[i] = g.tpos[i];
        if (pos[i] < 0) fixv[i] = (int)((base_amp >> g.q[i]) & 1);
    }
    int vb[2], nv = 0;  // matrix bits that vary inside the tile
    for (int i = 0; i < g.nq; ++i)
        if (pos[i] >= 0) vb[nv++] = i;
    int fixidx = 0;
    for (int i = 0; i < g.nq; ++i)
        if (pos[i] < 0) fixidx |= fixv[i] << i;
    auto M = [&](int r, int c) { return make_c<T, R>(g.m[2 * (r * dim + c)], g.m[2 * (r * dim + c) + 1]); };
    auto full = [&](int x) {  // matrix index of local pattern x
        int idx = fixidx;
        for (int k = 0; k < nv; ++k)
            if ((x >> k) & 1) idx |= 1 << vb[k];
        return idx;
    };
    const int size = 1 << nb;
    if (nv == 0) {
        const T c = M(fixidx, fixidx);
        for (int i = threadIdx.x; i < size; i += blockDim.x) t[i] = cmul(c, t[i]);
    } else if (nv == 1) {
        const int p = pos[vb[0]];
        const T e0 = M(full(0), full(0)), e1 = M(full(0), full(1)), e2 = M(full(1), full(0)), e3 = M(full(1), full(1));
        const int lowmask = (1 << p) - 1;
        for (int i = threadIdx.x; i < size / 2; i += blockDim.x) {
            const int i0 = ((i & ~lowmask) << 1) | (i & lowmask), i1 = i0 | (1 << p);
            const T a = t[i0], b = t[i1];
            t[i0] = cfma(e0, a, cmul(e1, b));
            t[i1] = cfma(e2, a, cmul(e3, b));
        }
    } else {
        const int pa = pos[0], pb = pos[1];
        const int lo = pa < pb ? pa : pb, hi = pa < pb ? pb : pa;
        const int mlo = (1 << lo) - 1, mhi = (1 << hi) - 1;
        T mm[16];
        for (int k = 0; k < 16; ++k) mm[k] = M(k / 4, k % 4);
        for (int i = threadIdx.x; i < size / 4; i += blockDim.x) {
            int b = ((i & ~mlo) << 1) | (i & mlo);
            b = ((b & ~mhi) << 1) | (b & mhi);
            const int ia = 1 << pa, ib = 1 << pb;
            const T v0 = t[b], v1 = t[b | ia], v2 = t[b | ib], v3 = t[b | ia | ib];
            T o[4];
            for (int r = 0; r < 4; ++r) {
                T acc = cmul(mm[4 * r], v0);
                acc = cfma(mm[4 * r + 1], v1, acc);
                acc = cfma(mm[4 * r + 2], v2, acc);
                acc = cfma(mm[4 * r + 3], v3, acc);
                o[r] = acc;
            }
            t[b] = o[0];
            t[b | ia] = o[1];
            t[b | ib] = o[2];
            t[b | ia | ib] = o[3];
        }
    }
}

constexpr int kAdjThreads = 256;
constexpr int kMaxAdjSlots = 128;

template <typename R, int RB>
__device__ void dual_tile_sweeps(typename Cplx<R>::T *tA, typename Cplx<R>::T *tB, int nb, const Sweep *__restrict__ sweeps,
                                 int nsweeps, const ROp *__restrict__ ops, const typename Cplx<R>::T *__restrict__ pool,
                                 uint32_t ow, double *s_acc, int lane);

// kC, kJ: the chunk and tile-qubit counts as compile-time constants (0 = read
// them from the launch arguments).
template <typename R, int kC, int kJ>
__global__ void __launch_bounds__(kAdjThreads, 2) adjoint_pass_kernel(const AdjPassArgs a) {
    using T = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double s_acc[2 * kMaxAdjSlots];
    __shared__ int32_t s_tq[kMaxTileQubits];
    const int C = kC ? kC : a.C, j = kJ ? kJ : a.j, nb = C + j, size = 1 << nb;
    const int cmask = (1 << C) - 1;
    const int lane = threadIdx.x & 31;
    T *tp = reinterpret_cast<T *>(smem);
    T *tl = tp + size;
    T *psi = reinterpret_cast<T *>(a.psi);
    T *lam = reinterpret_cast<T *>(a.lam);
    for (int i = threadIdx.x; i < 2 * a.nslots; i += blockDim.x) s_acc[i] = 0.0;
    if (threadIdx.x < kMaxTileQubits) s_tq[threadIdx.x] = a.tq[threadIdx.x];
    __syncthreads();
    for (uint64_t tile_id = blockIdx.x; tile_id < a.n_tiles; tile_id += gridDim.x) {
        const uint64_t chunk_base = insert_zero_bits(tile_id, s_tq, j);
        for (int e = threadIdx.x; e < size; e += blockDim.x) {
            const uint64_t amp = ((chunk_base | deposit_bits((uint32_t)(e >> C), s_tq, j)) << C) | (uint64_t)(e & cmask);
            tp[e] = psi[amp];
            tl[e] = lam[amp];
        }
        __syncthreads();
        const uint64_t base_amp = chunk_base << C;
        if (a.nsweeps > 0) {
            uint32_t ow = 0;
            for (int i = 0; i < a.nouter; ++i) ow |= (uint32_t)((base_amp >> a.outer_q[i]) & 1u) << i;
            if constexpr (sizeof(R) == 4)
                dual_tile_sweeps<R, kDualRegBitsF32>(tp, tl, nb, a.sweeps, a.nsweeps, a.rops,
                                                     reinterpret_cast<const T *>(a.pool), ow, s_acc, lane);
            else
                dual_tile_sweeps<R, kDualRegBitsF64>(tp, tl, nb, a.sweeps, a.nsweeps, a.rops,
                                                     reinterpret_cast<const T *>(a.pool), ow, s_acc, lane);
        }
        for (int k = 0; k < (a.nsweeps > 0 ? 0 : a.ngates); ++k) {
            const AdjGate &ag = a.gates[k];
            if (ag.slot >= 0) {
                const int outer = __popcll(base_amp & ag.gen.zo) & 1;
                double re = 0.0, im = 0.0;
                for (int x = threadIdx.x; x < size; x += blockDim.x) {
                    const T ax = tp[x];
                    const T by = tl[x ^ (int)ag.gen.xt];
                    double pr = (double)by.x * (double)ax.x + (double)by.y * (double)ax.y;
                    double pi = (double)by.x * (double)ax.y - (double)by.y * (double)ax.x;
                    if ((__popc((uint32_t)x & ag.gen.zt) + outer) & 1) { pr = -pr; pi = -pi; }
                    re += pr;
                    im += pi;
                }
                re = block_warp_sum(re);
                im = block_warp_sum(im);
                if (lane == 0) {
                    atomicAdd(&s_acc[2 * ag.slot], re);
                    atomicAdd(&s_acc[2 * ag.slot + 1], im);
                }
                __syncthreads();
            }
            smem_apply_gate<R>(tp, nb, ag.g, base_amp);
            smem_apply_gate<R>(tl, nb, ag.g, base_amp);
            __syncthreads();
        }
        for (int e = threadIdx.x; e < size; e += blockDim.x) {
            const uint64_t amp = ((chunk_base | deposit_bits((uint32_t)(e >> C), s_tq, j)) << C) | (uint64_t)(e & cmask);
            psi[amp] = tp[e];
            lam[amp] = tl[e];
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < 2 * a.nslots; i += blockDim.x)
        if (s_acc[i] != 0.0) atomicAdd(&a.out[i], s_acc[i]);
}

// ------------------------------------------------------------ dual-store pass
// One pass over two compressed stores A and B (DualPassArgs): both tiles are
// decoded into shared memory (linear layout), the op list runs in order
// (gates with smem_apply_gate, transition sums, Pauli-term accumulation into
// B), and each written store is re-encoded into its output arena with one
// reservation per tile.  Blocks not stored at the start of the pass read as
// zeros; every chunk of a written store is written.
// Threads of a two-store pass CTA: 8 warps for tiles of 2^12 amplitudes (two
// CTAs per SM), 16 warps for 2^13-amplitude complex64 tiles, whose two value
// tiles (128 KB) leave room for one CTA per SM.
constexpr int kDualThreads = 256;
constexpr int kDualThreadsWide = 512;
inline int dual_threads(int nb) { return nb >= 13 ? kDualThreadsWide : kDualThreads; }

template <typename R>
__device__ void dual_decode_tile(const DualStore &st, int C, int j, int blk_shift, uint64_t chunk_base,
                                 const int32_t *s_tq, CodecParams p, R *tile, uint32_t *wstage, int warp, int nwarps,
                                 int lane) {
    const int nchunks = 1 << j, ncomp = 2 << C, per_lane = ncomp >> 5;
    for (int c = warp; c < nchunks; c += nwarps) {
        R *comp = tile + (size_t)c * ncomp;
        const uint64_t chunk = chunk_base | deposit_bits((uint32_t)c, s_tq, j);
        if (st.meta_in == nullptr || !st.mask_in[chunk >> blk_shift]) {
            for (int i = 0; i < per_lane; ++i) comp[lane + 32 * i] = R(0);
            continue;
        }
        decode_chunk<R>(st.arena_in, st.meta_in[chunk], per_lane, p, comp, wstage, lane);
        __syncwarp();
    }
}

// Quantise, reserve and pack one store's tile (codes overwrite the values).
template <typename R>
__device__ bool dual_encode_tile(const DualStore &st, int C, int j, int blk_shift, uint64_t chunk_base,
                                 const int32_t *s_tq, CodecParams p, R *tile, int32_t *s_base, uint32_t *s_width,
                                 unsigned long long *s_off, unsigned long long *s_tile_off, int *s_flag,
                                 int32_t *error, int warp, int nwarps, int lane) {
    const int nchunks = 1 << j, ncomp = 2 << C, per_lane = ncomp >> 5;
    for (int c = warp; c < nchunks; c += nwarps) {
        R *comp = tile + (size_t)c * ncomp;
        int32_t base;
        uint32_t width;
        bool nz;
        quantize_chunk<R>(comp, per_lane, p, false, lane, &base, &width, &nz);
        if (lane == 0) {
            s_base[c] = base;
            s_width[c] = width;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int c = 0; c < nchunks; ++c) {
            s_off[c] = run;
            run += payload_bytes(C, s_width[c]);
        }
        const unsigned long long off = atomicAdd(st.bump, run);
        *s_flag = 0;
        if (off + run > st.capacity) {
            atomicExch(error, 1);
            *s_flag = 1;
        }
        *s_tile_off = off;
    }
    __syncthreads();
    if (*s_flag) return false;
    for (int c = warp; c < nchunks; c += nwarps) {
        const uint64_t chunk = chunk_base | deposit_bits((uint32_t)c, s_tq, j);
        const int32_t *codes = reinterpret_cast<const int32_t *>(tile + (size_t)c * ncomp);
        const unsigned long long off = *s_tile_off + s_off[c];
        const uint32_t w = s_width[c];
        pack_chunk(codes, per_lane, s_base[c], w, st.arena_out + (off >> 2), lane);
        if (lane == 0) {
            ChunkMeta md;
            md.offset = off;
            md.base = s_base[c];
            md.width = w;
            st.meta_out[chunk] = md;
            atomicAdd(&st.block_bytes[chunk >> blk_shift],
                      (unsigned long long)(payload_bytes(C, w) + sizeof(ChunkMeta)));
        }
    }
    __syncthreads();
    return true;
}

// sum_s conj(w[s ^ X]) (-1)^{|s & zs|} v[s] over a register group, X a
// compile-time flip mask (the caller dispatches on the op's mask).
template <int NS, int X, typename T>
__device__ __forceinline__ void group_pauli_sum(const T (&v)[NS], const T (&w)[NS], int zs, double &re, double &im) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const T a = v[s], b = w[s ^ X];
        double pr = (double)b.x * (double)a.x + (double)b.y * (double)a.y;
        double pi = (double)b.x * (double)a.y - (double)b.y * (double)a.x;
        const double sg = (__popc(s & zs) & 1) ? -1.0 : 1.0;
        re = fma(sg, pr, re);
        im = fma(sg, pi, im);
    }
}

template <int RB, typename T>
__device__ __forceinline__ void group_pauli_sum_any(const T (&v)[1 << RB], const T (&w)[1 << RB], int xs, int zs,
                                                    double &re, double &im) {
    constexpr int NS = 1 << RB;
#define QS_GS(X) \
    case X:      \
        if constexpr ((X) < NS) group_pauli_sum<NS, (X)>(v, w, zs, re, im); \
        break;
    switch (xs) {
        QS_GS(0) QS_GS(1) QS_GS(2) QS_GS(3) QS_GS(4) QS_GS(5) QS_GS(6) QS_GS(7)
        QS_GS(8) QS_GS(9) QS_GS(10) QS_GS(11) QS_GS(12) QS_GS(13) QS_GS(14) QS_GS(15)
        default: break;
    }
#undef QS_GS
}

// Register sweeps over the two tiles of a two-store pass: each thread holds
// the group of store A (v) and the group of store B (w) at the same 2^RB tile
// positions, applies every gate op of the sweep to both, and at each OPC_SUM
// adds the group's share of the derivative sum to s_acc (warp sums, one
// shared-memory atomic per warp).  Tiles are in the linear layout.  The
// group loop runs the same trip count in every warp, so that the warp sums
// see all 32 lanes.
template <typename R, int RB>
__device__ void dual_tile_sweeps(typename Cplx<R>::T *tA, typename Cplx<R>::T *tB, int nb, const Sweep *__restrict__ sweeps,
                                 int nsweeps, const ROp *__restrict__ ops, const typename Cplx<R>::T *__restrict__ pool,
                                 uint32_t ow, double *s_acc, int lane) {
    using T = typename Cplx<R>::T;
    constexpr int NS = 1 << RB;
    const int groups = 1 << (nb - RB);
    const uint32_t wo = ow << nb;
    for (int sidx = 0; sidx < nsweeps; ++sidx) {
        const Sweep sw = sweeps[sidx];
        int sb[RB], bm[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            sb[k] = sw.sbits[k];
            bm[k] = 1 << sb[k];
        }
        auto off = [&](int s) {
            int o = 0;
#pragma unroll
            for (int k = 0; k < RB; ++k)
                if ((s >> k) & 1) o |= bm[k];
            return o;
        };
        for (int g0 = 0; g0 < groups; g0 += blockDim.x) {
            const int grp = g0 + threadIdx.x;
            const bool live = grp < groups;
            int base = live ? grp : 0;
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                const int t = sb[k];
                base = ((base >> t) << (t + 1)) | (base & ((1 << t) - 1));
            }
            const uint32_t W = (uint32_t)base | wo;
            T v[NS], w[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                v[s] = live ? tA[base | off(s)] : make_c<T, R>(0.0, 0.0);
                w[s] = live ? tB[base | off(s)] : make_c<T, R>(0.0, 0.0);
            }
            T za = c_one<T>(), zb = c_one<T>(), zha = c_one<T>(), zhb = c_one<T>();
            for (int k = sw.g0; k < sw.g1; ++k) {
                const ROp o = ops[k];
                if (o.code == OPC_SUM) {
                    const T f = pool[o.mat + rop_variant(o, W)];
                    double re = 0.0, im = 0.0;
                    group_pauli_sum_any<RB>(v, w, o.pad >> 4, o.pad & 15, re, im);
                    // conj(zb) za f (re + i im)
                    const double cr = (double)zb.x * (double)za.x + (double)zb.y * (double)za.y;
                    const double ci = (double)zb.x * (double)za.y - (double)zb.y * (double)za.x;
                    const double fr = (double)f.x;
                    double sr = fr * (cr * re - ci * im), si = fr * (cr * im + ci * re);
#pragma unroll
                    for (int d = 16; d > 0; d >>= 1) {
                        sr += __shfl_xor_sync(0xffffffffu, sr, d);
                        si += __shfl_xor_sync(0xffffffffu, si, d);
                    }
                    if (lane == 0) {
                        atomicAdd(&s_acc[2 * o.vstride], sr);
                        atomicAdd(&s_acc[2 * o.vstride + 1], si);
                    }
                } else {
                    const T *m = pool + o.mat + rop_variant(o, W) * o.vstride;
                    apply_rop<RB>(v, za, zha, o.code, m);
                    apply_rop<RB>(w, zb, zhb, o.code, m);
                }
            }
            if (live) {
                const bool sa = za.x != R(1) || za.y != R(0), sbz = zb.x != R(1) || zb.y != R(0);
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    tA[base | off(s)] = sa ? cmul(za, v[s]) : v[s];
                    tB[base | off(s)] = sbz ? cmul(zb, w[s]) : w[s];
                }
            }
        }
        __syncthreads();
    }
}

// kC, kJ: chunk log2 and tile qubits above the chunk as compile-time
// constants (0: read from the args), as for pass_kernel.
template <typename R, int kC, int kJ>
__global__ void __launch_bounds__(kDualThreadsWide) dual_pass_kernel(const DualPassArgs a) {
    using T = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char dual_smem[];
    __shared__ double s_acc[2 * kMaxDualSlots];
    __shared__ int32_t s_tq[kMaxTileQubits];
    __shared__ unsigned long long s_tile_off;
    __shared__ int s_flag;
    const int C = kC ? kC : a.C, j = kJ ? kJ : a.j, nb = C + j, size = 1 << nb;
    const int nchunks = 1 << j;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int blk_shift = a.B - C;
    T *tA = reinterpret_cast<T *>(dual_smem);
    T *tB = tA + size;
    uint32_t *wstage = reinterpret_cast<uint32_t *>(tB + size) + warp * kStageWords;
    int32_t *s_base = reinterpret_cast<int32_t *>(reinterpret_cast<uint32_t *>(tB + size) + nwarps * kStageWords);
    uint32_t *s_width = reinterpret_cast<uint32_t *>(s_base + nchunks);
    unsigned long long *s_off = reinterpret_cast<unsigned long long *>(s_base + 2 * nchunks);  // 8-byte aligned
    for (int i = threadIdx.x; i < 2 * a.nslots; i += blockDim.x) s_acc[i] = 0.0;
    if (threadIdx.x < kMaxTileQubits) s_tq[threadIdx.x] = a.tq[threadIdx.x];
    __syncthreads();
    for (uint64_t tile_id = blockIdx.x; tile_id < a.n_tiles; tile_id += gridDim.x) {
        const uint64_t chunk_base = insert_zero_bits(tile_id, s_tq, j);
        const uint64_t base_amp = chunk_base << C;
        dual_decode_tile<R>(a.a, C, j, blk_shift, chunk_base, s_tq, a.codec, reinterpret_cast<R *>(tA), wstage,
                            warp, nwarps, lane);
        dual_decode_tile<R>(a.b, C, j, blk_shift, chunk_base, s_tq, a.codec, reinterpret_cast<R *>(tB), wstage,
                            warp, nwarps, lane);
        __syncthreads();
        if (a.nsweeps > 0) {
            uint32_t ow = 0;
            for (int i = 0; i < a.nouter; ++i) ow |= (uint32_t)((base_amp >> a.outer_q[i]) & 1u) << i;
            if constexpr (sizeof(R) == 4)
                dual_tile_sweeps<R, kDualRegBitsF32>(tA, tB, nb, a.sweeps, a.nsweeps, a.rops,
                                                     reinterpret_cast<const T *>(a.pool), ow, s_acc, lane);
            else
                dual_tile_sweeps<R, kDualRegBitsF64>(tA, tB, nb, a.sweeps, a.nsweeps, a.rops,
                                                     reinterpret_cast<const T *>(a.pool), ow, s_acc, lane);
        }
        for (int k = 0; k < (a.nsweeps > 0 ? 0 : a.nops); ++k) {
            const DualOp &op = a.ops[k];
            if (op.kind == DOP_SUM) {
                const int outer = __popcll(base_amp & op.term.zo) & 1;
                double re = 0.0, im = 0.0;
                for (int x = threadIdx.x; x < size; x += blockDim.x) {
                    const T ax = tA[x];
                    const T by = tB[x ^ (int)op.term.xt];
                    double pr = (double)by.x * (double)ax.x + (double)by.y * (double)ax.y;
                    double pi = (double)by.x * (double)ax.y - (double)by.y * (double)ax.x;
                    if ((__popc((uint32_t)x & op.term.zt) + outer) & 1) { pr = -pr; pi = -pi; }
                    re += pr;
                    im += pi;
                }
                re = block_warp_sum(re);
                im = block_warp_sum(im);
                if (lane == 0) {
                    atomicAdd(&s_acc[2 * op.slot], re);
                    atomicAdd(&s_acc[2 * op.slot + 1], im);
                }
            } else if (op.kind == DOP_ACCUM) {
                const int outer = __popcll(base_amp & op.term.zo) & 1;
                const double cr = op.coef[0], ci = op.coef[1];
                for (int x = threadIdx.x; x < size; x += blockDim.x) {
                    const int y = x ^ (int)op.term.xt;
                    const T v = tA[y];
                    const double sg = ((__popc((uint32_t)y & op.term.zt) + outer) & 1) ? -1.0 : 1.0;
                    T &o = tB[x];
                    o.x = (R)((double)o.x + sg * (cr * (double)v.x - ci * (double)v.y));
                    o.y = (R)((double)o.y + sg * (cr * (double)v.y + ci * (double)v.x));
                }
            } else {
                if (op.kind != DOP_GATE_B) smem_apply_gate<R>(tA, nb, op.g, base_amp);
                if (op.kind != DOP_GATE_A) smem_apply_gate<R>(tB, nb, op.g, base_amp);
            }
            __syncthreads();
        }
        if (a.a.meta_out &&
            !dual_encode_tile<R>(a.a, C, j, blk_shift, chunk_base, s_tq, a.codec, reinterpret_cast<R *>(tA), s_base,
                                 s_width, s_off, &s_tile_off, &s_flag, a.error, warp, nwarps, lane))
            break;
        if (!dual_encode_tile<R>(a.b, C, j, blk_shift, chunk_base, s_tq, a.codec, reinterpret_cast<R *>(tB), s_base,
                                 s_width, s_off, &s_tile_off, &s_flag, a.error, warp, nwarps, lane))
            break;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * a.nslots; i += blockDim.x)
        if (s_acc[i] != 0.0) atomicAdd(&a.sums[i], s_acc[i]);
}

size_t dual_pass_smem_bytes(bool f64, int C, int j) {
    const size_t nch = (size_t)1 << j;
    // two value tiles, the warps' staging areas, then base, width and offset per chunk
    return ((size_t)2 * (f64 ? 16 : 8) << (C + j)) + (size_t)(dual_threads(C + j) / 32) * kStageWords * 4 + 16 * nch;
}

// Imported stores: the header of every chunk of an unstored block is set to
// zero (offset 0, width 0), so that a reader that skipped the zero-mask gate
// would still read inside the arena.
__global__ void zero_unstored_headers_kernel(ChunkMeta *meta, const uint8_t *mask, uint64_t nchunks, int cshift) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nchunks;
         k += (uint64_t)gridDim.x * blockDim.x)
        if (!mask[k >> cshift]) meta[k] = ChunkMeta{0, 0, 0};
}

// ------------------------------------------------------------ chunk exchange
// Chunk index of half index k: bit `bit` of the chunk index set to v.
__device__ __forceinline__ uint64_t half_chunk(uint64_t k, int bit, uint32_t v) {
    const uint64_t lo = k & ((uint64_t(1) << bit) - 1);
    return ((k >> bit) << (bit + 1)) | ((uint64_t)v << bit) | lo;
}

__global__ void half_sizes_kernel(const HalfChunks h, const ChunkMeta *meta, const uint8_t *mask, uint64_t *sizes,
                                  uint8_t *flags) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < h.nhalf;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = half_chunk(k, h.bit, h.value);
        const bool st = mask[c >> h.cshift] != 0;
        const uint32_t w = st ? min(meta[c].width, 32u) : 0u;
        sizes[k] = st ? payload_bytes(h.C, w) : 0;
        flags[k] = st ? 1 : 0;
    }
}

// Block-wide inclusive sum of one value per thread (blockDim.x = 1024).
__device__ __forceinline__ uint64_t block_inclusive_scan(uint64_t x, uint64_t *s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t y = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        s_warp[lane] = y;
    }
    __syncthreads();
    const uint64_t r = x + (warp > 0 ? s_warp[warp - 1] : 0);
    __syncthreads();
    return r;
}

constexpr int kScanThreads = 1024, kScanPerThread = 4, kScanPerBlock = kScanThreads * kScanPerThread;

// Per-CTA exclusive scan of kScanPerBlock values in place; the CTA's total to totals[cta].
__global__ void __launch_bounds__(kScanThreads) half_scan_blocks_kernel(uint64_t *v, uint64_t n, uint64_t *totals) {
    __shared__ uint64_t s_warp[32];
    const uint64_t i0 = (uint64_t)blockIdx.x * kScanPerBlock + (uint64_t)threadIdx.x * kScanPerThread;
    uint64_t a[kScanPerThread], sum = 0;
#pragma unroll
    for (int t = 0; t < kScanPerThread; ++t) {
        a[t] = i0 + t < n ? v[i0 + t] : 0;
        sum += a[t];
    }
    const uint64_t incl = block_inclusive_scan(sum, s_warp);
    uint64_t run = incl - sum;
#pragma unroll
    for (int t = 0; t < kScanPerThread; ++t) {
        if (i0 + t < n) v[i0 + t] = run;
        run += a[t];
    }
    if (threadIdx.x == blockDim.x - 1) totals[blockIdx.x] = incl;
}

// One CTA: exclusive scan of the m CTA totals in place, grand total to *total.
__global__ void __launch_bounds__(kScanThreads) half_scan_totals_kernel(uint64_t *totals, uint64_t m, uint64_t *total) {
    __shared__ uint64_t s_warp[32];
    const uint64_t per = (m + kScanThreads - 1) / kScanThreads;
    const uint64_t i0 = (uint64_t)threadIdx.x * per;
    uint64_t sum = 0;
    for (uint64_t i = i0; i < i0 + per && i < m; ++i) sum += totals[i];
    const uint64_t incl = block_inclusive_scan(sum, s_warp);
    uint64_t run = incl - sum;
    for (uint64_t i = i0; i < i0 + per && i < m; ++i) {
        const uint64_t t = totals[i];
        totals[i] = run;
        run += t;
    }
    if (threadIdx.x == blockDim.x - 1) *total = incl;
}

__global__ void half_scan_add_kernel(uint64_t *v, uint64_t n, const uint64_t *totals) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        v[i] += totals[i / kScanPerBlock];
}

// One warp per half chunk: its packed header, then its payload copied in
// 16-byte words (payloads are 128-byte aligned on both sides).
__global__ void half_pack_kernel(const HalfChunks h, const ChunkMeta *meta, const uint32_t *arena,
                                 const uint8_t *flags, const uint64_t *offsets, ChunkMeta *out_meta,
                                 uint32_t *out_payload, bool scatter) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; k < h.nhalf; k += warps) {
        const uint64_t c = half_chunk(k, h.bit, h.value);
        ChunkMeta md{0, 0, 0};
        if (flags[k]) {
            md = meta[c];
            md.width = min(md.width, 32u);
        }
        const uint64_t bytes = flags[k] ? payload_bytes(h.C, md.width) : 0;
        const uint4 *src = reinterpret_cast<const uint4 *>(arena + (md.offset >> 2));
        uint4 *dst = reinterpret_cast<uint4 *>(out_payload + (offsets[k] >> 2));
        for (uint64_t w = lane; w < bytes / 16; w += 32) dst[w] = src[w];
        if (lane == 0)
            out_meta[scatter ? c : k] = flags[k] ? ChunkMeta{offsets[k], md.base, md.width} : ChunkMeta{0, 0, 0};
    }
}

__global__ void half_unpack_kernel(const HalfChunks h, const ChunkMeta *in_meta, const uint8_t *in_flags,
                                   uint64_t base, ChunkMeta *meta, uint8_t *mask) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < h.nhalf;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = half_chunk(k, h.bit, h.value);
        ChunkMeta md = in_meta[k];
        if (in_flags[k]) {
            md.offset += base;
            md.width = min(md.width, 32u);
            mask[c >> h.cshift] = 1;
        } else {
            md = ChunkMeta{0, 0, 0};
            // a block-level qubit moves whole blocks: an unstored one stays unstored
            if (h.bit >= h.cshift) mask[c >> h.cshift] = 0;
        }
        meta[c] = md;
    }
}

// Received headers: stored chunks must have a 128-byte aligned offset, a
// width of at most 32 and a payload inside the received payload bytes.
__global__ void half_check_kernel(const HalfChunks h, const ChunkMeta *in_meta, const uint8_t *in_flags,
                                  uint64_t payload_bytes_total, int32_t *bad) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < h.nhalf;
         k += (uint64_t)gridDim.x * blockDim.x) {
        if (!in_flags[k]) continue;
        const ChunkMeta md = in_meta[k];
        const uint64_t pb = payload_bytes(h.C, md.width & 63u);
        if (md.width > 32 || (md.offset & 127) || md.offset > payload_bytes_total || pb > payload_bytes_total - md.offset)
            atomicOr(bad, 1);
    }
}

// One warp per block.
__global__ void block_bytes_kernel(const ChunkMeta *meta, const uint8_t *mask, uint32_t nb, int cshift, int C,
                                   unsigned long long *block_bytes) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t cpb = uint64_t(1) << cshift;
    for (uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; b < nb; b += warps) {
        unsigned long long s = 0;
        if (mask[b])
            for (uint64_t k = lane; k < cpb; k += 32)
                s += payload_bytes(C, min(meta[(b << cshift) + k].width, 32u)) + sizeof(ChunkMeta);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) block_bytes[b] = mask[b] ? s : 0;
    }
}

// Raises a kernel's dynamic shared-memory limit to at least `smem` bytes on
// the current device and never lowers it: the limit is per function, shared
// by every host thread and handle, so a thread that lowered it between
// another thread's setting and its launch would make that launch fail.
std::mutex g_smem_attr_mu;
std::map<std::pair<const void *, int>, size_t> g_smem_attr;

template <typename K>
cudaError_t ensure_dyn_smem(K *kernel, size_t smem) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_smem_attr_mu);
    size_t &cur = g_smem_attr[{reinterpret_cast<const void *>(kernel), dev}];
    if (smem <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) cur = smem;
    return e;
}

int g_sm_count = 0;

// Scratch of the allocation-free codec round trip (qs_codec_roundtrip_noalloc):
// the packed words between encode and decode.  Every GPU that loads the
// library holds these 4 MiB until the process exits.
constexpr uint64_t kNoAllocScratchWords = uint64_t(1) << 20;
static __device__ __align__(256) uint32_t g_noalloc_words[kNoAllocScratchWords];

unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap_per_sm = 8) {
    const uint64_t need = (work + per_block - 1) / per_block;
    const uint64_t cap = (uint64_t)sm_count() * cap_per_sm;
    uint64_t g = need < cap ? need : cap;
    return (unsigned)(g ? g : 1);
}

}  // namespace

int sm_count() {
    if (g_sm_count == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        g_sm_count = v;
    }
    return g_sm_count;
}

template <typename R, int RB, bool kCodes, int kHB, int kC, int kJ>
static cudaError_t launch_pass_kc(const PassArgs &a, cudaStream_t s) {
    const int nb = a.C + a.j;
    const size_t smem = pass_smem_bytes(sizeof(R) == 8, nb, a.j);
    cudaError_t e = ensure_dyn_smem(pass_kernel<R, RB, kCodes, kHB, kC, kJ>, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass_kernel<R, RB, kCodes, kHB, kC, kJ>, kSweepThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid == 0) grid = 1;
    // arena slabs per CTA when the arena can spare 8 of them per CTA
    PassArgs b = a;
    const char *env = std::getenv("QOMPSIM_SLAB_BYTES");
    const uint64_t slab = env ? (uint64_t)std::strtoull(env, nullptr, 10) : (uint64_t)kArenaSlabBytes;
    b.slab = (slab && a.capacity / grid >= 8 * slab) ? (slab + 127) / 128 * 128 : 0;
    pass_kernel<R, RB, kCodes, kHB, kC, kJ><<<(unsigned)grid, kSweepThreads, smem, s>>>(b);
    return cudaGetLastError();
}

// The default chunk size (2^8 amplitudes) and the default tile (2^12
// amplitudes for complex128, 2^13 for complex64, i.e. 4 or 5 tile qubits
// above the chunk) are compile-time constants of their instantiation: the
// per-lane counts, chunk and group counts, offsets and swizzle mask then fold
// into the code (measured 12-19 % faster than reading them from the args).
template <typename R, int RB, bool kCodes, int kHB>
static cudaError_t launch_pass_t(const PassArgs &a, cudaStream_t s) {
    constexpr int J = sizeof(R) == 8 ? 4 : 5;
    if (a.C == kMaxChunkLog2 && a.j == J) return launch_pass_kc<R, RB, kCodes, kHB, kMaxChunkLog2, J>(a, s);
    return a.C == kMaxChunkLog2 ? launch_pass_kc<R, RB, kCodes, kHB, kMaxChunkLog2, 0>(a, s)
                                : launch_pass_kc<R, RB, kCodes, kHB, 0, 0>(a, s);
}

template <typename R, bool kCodes, bool kDense, int kC, int kJ>
static cudaError_t launch_staged_kc(const PassArgs &a, cudaStream_t s) {
    const uint32_t nblk = 1u << (a.n - a.B);
    const uint32_t mask_words = nblk <= kMaxSmemBlocks ? (nblk + 31) / 32 : 0;
    const size_t smem = staged_layout(sizeof(R) == 8, a.C, a.j, mask_words, kDense ? a.dense.k : 0).total;
    cudaError_t e = ensure_dyn_smem(staged_pass_kernel<R, kCodes, kDense, kC, kJ>, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, staged_pass_kernel<R, kCodes, kDense, kC, kJ>, kStagedThreads,
                                                      smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid == 0) grid = 1;
    PassArgs b = a;
    const char *env = std::getenv("QOMPSIM_SLAB_BYTES");
    const uint64_t slab = env ? (uint64_t)std::strtoull(env, nullptr, 10) : (uint64_t)kArenaSlabBytes;
    b.slab = (slab && a.capacity / grid >= 8 * slab) ? (slab + 127) / 128 * 128 : 0;
    staged_pass_kernel<R, kCodes, kDense, kC, kJ><<<(unsigned)grid, kStagedThreads, smem, s>>>(b);
    return cudaGetLastError();
}

size_t staged_pass_smem_bytes(bool f64, int C, int j, uint32_t nblocks) {
    return staged_layout(f64, C, j, nblocks <= kMaxSmemBlocks ? (nblocks + 31) / 32 : 0).total;
}

template <typename R, bool kCodes, bool kDense = false>
static cudaError_t launch_staged_t(const PassArgs &a, cudaStream_t s) {
    if (a.C == kMaxChunkLog2 && a.C + a.j == kDenseTileLog2)
        return launch_staged_kc<R, kCodes, kDense, kMaxChunkLog2, kDenseTileLog2 - kMaxChunkLog2>(a, s);
    return launch_staged_kc<R, kCodes, kDense, 0, 0>(a, s);
}

cudaError_t launch_pass(bool f64, const PassArgs &a, int, cudaStream_t s) {
    if (a.rb != kRegBits || a.C + a.j < kRegBits || a.diag.nterms > kMaxDiagTerms) return cudaErrorInvalidValue;
    if (a.code_moves && a.diag.nterms) return cudaErrorInvalidValue;
    if (a.header_batch != 4 && a.header_batch != 8) return cudaErrorInvalidValue;
    if (a.dense.k) {
        // one dense k-qubit gate over 2^kDenseTileLog2-amplitude tiles (staged kernel only)
        if (a.dense.k < kMinDenseK || a.dense.k > kMaxDenseK || a.C + a.j != kDenseTileLog2 || a.code_moves ||
            a.diag.nterms || !a.staged)
            return cudaErrorInvalidValue;
        for (int i = 0; i < a.dense.k; ++i)
            if (a.dense.pos[i] < 0 || a.dense.pos[i] >= kDenseTileLog2) return cudaErrorInvalidValue;
        return f64 ? launch_staged_t<double, false, true>(a, s) : launch_staged_t<float, false, true>(a, s);
    }
    if (a.staged) {
        if (f64) return a.code_moves ? launch_staged_t<double, true>(a, s) : launch_staged_t<double, false>(a, s);
        return a.code_moves ? launch_staged_t<float, true>(a, s) : launch_staged_t<float, false>(a, s);
    }
    if (f64)
        return a.code_moves ? launch_pass_t<double, kRegBits, true, 4>(a, s) : launch_pass_t<double, kRegBits, false, 4>(a, s);
    if (a.code_moves)
        return a.header_batch == 8 ? launch_pass_t<float, kRegBits, true, 8>(a, s)
                                   : launch_pass_t<float, kRegBits, true, 4>(a, s);
    return a.header_batch == 8 ? launch_pass_t<float, kRegBits, false, 8>(a, s)
                               : launch_pass_t<float, kRegBits, false, 4>(a, s);
}

cudaError_t launch_perm_pass(const PermPassArgs &a, cudaStream_t s) {
    const unsigned grid = grid_for(a.nchunks, 256, 16);
    perm_pass_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename R, int RB, int kC, int kJ>
static cudaError_t launch_dense_pass_kc(const DensePassArgs &a, cudaStream_t s) {
    const int nb = a.C + a.j;
    const size_t smem = (size_t)(2 * sizeof(R)) << nb;
    auto kern = dense_pass_kernel<R, RB, kC, kJ>;
    cudaError_t e = ensure_dyn_smem(kern, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSweepThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid == 0) grid = 1;
    kern<<<(unsigned)grid, kSweepThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// The uncompressed fused path's default geometry: 2^5-amplitude chunks and
// tiles of 2^12 (complex128) or 2^13 (complex64) amplitudes.
template <typename R, int RB>
static cudaError_t launch_dense_pass_t(const DensePassArgs &a, cudaStream_t s) {
    constexpr int kDC = 5, kDJ = sizeof(R) == 8 ? 7 : 8;
    if (a.C == kDC && a.j == kDJ) return launch_dense_pass_kc<R, RB, kDC, kDJ>(a, s);
    return launch_dense_pass_kc<R, RB, 0, 0>(a, s);
}

cudaError_t launch_dense_pass(bool f64, const DensePassArgs &a, int, cudaStream_t s) {
    if (a.rb != kRegBits || a.C + a.j < kRegBits) return cudaErrorInvalidValue;
    return f64 ? launch_dense_pass_t<double, kRegBits>(a, s) : launch_dense_pass_t<float, kRegBits>(a, s);
}

cudaError_t launch_pergate(bool f64, void *state, int n, const KGate *g, cudaStream_t s) {
    const uint64_t work = uint64_t(1) << (n - 1);
    const unsigned grid = grid_for(work, 256, 16);
    if (f64) pergate_kernel<double><<<grid, 256, 0, s>>>((double2 *)state, n, g);
    else pergate_kernel<float><<<grid, 256, 0, s>>>((float2 *)state, n, g);
    return cudaGetLastError();
}

cudaError_t launch_stage_begin(const uint32_t *b2g, const uint8_t *mask, uint32_t nb, uint8_t *group_active,
                               uint32_t num_groups, uint32_t *block_nz, unsigned long long *block_bytes,
                               unsigned long long *active_blocks, cudaStream_t s) {
    const uint32_t m = nb > num_groups ? nb : num_groups;
    stage_clear_kernel<<<(m + 255) / 256, 256, 0, s>>>(group_active, num_groups, block_nz, block_bytes, nb);
    stage_mark_kernel<<<(nb + 255) / 256, 256, 0, s>>>(b2g, mask, nb, group_active);
    stage_count_kernel<<<(nb + 255) / 256, 256, 0, s>>>(b2g, group_active, nb, active_blocks);
    return cudaGetLastError();
}

cudaError_t launch_stage_end(const uint32_t *b2g, const uint8_t *group_active, uint32_t nb, const uint32_t *block_nz,
                             const unsigned long long *acc, uint8_t *mask, unsigned long long *block_bytes,
                             unsigned long long *history_slot, cudaStream_t s) {
    stage_end_kernel<<<(nb + 255) / 256, 256, 0, s>>>(b2g, group_active, nb, block_nz, acc, mask, block_bytes,
                                                      history_slot);
    return cudaGetLastError();
}

cudaError_t launch_mask_full(const uint8_t *mask, uint32_t nb, uint32_t *out, cudaStream_t s) {
    uint32_t grid = (nb + 1023u) / 1024u;
    grid = grid > 148u ? 148u : (grid ? grid : 1u);
    mask_full_kernel<<<grid, 1024, 0, s>>>(mask, nb, out);
    return cudaGetLastError();
}

cudaError_t launch_readback(const ReadbackList &l, unsigned long long *dst, cudaStream_t s) {
    if (l.n < 0 || l.n > 4) return cudaErrorInvalidValue;
    readback_kernel<<<1, 256, 0, s>>>(l, dst);
    return cudaGetLastError();
}

cudaError_t launch_sum_mask_bytes(const uint8_t *mask, const unsigned long long *bb, uint32_t nb,
                                  unsigned long long *out, cudaStream_t s) {
    sum_mask_bytes_kernel<<<(nb + 255) / 256, 256, 0, s>>>(mask, bb, nb, out);
    return cudaGetLastError();
}

cudaError_t launch_readout(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B, int C,
                           CodecParams p, uint64_t chunk0, uint64_t nchunks, double *out, double scale,
                           cudaStream_t s) {
    const unsigned grid = grid_for(nchunks, kPassThreads / 32, 8);
    if (f64) readout_kernel<double><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, chunk0, nchunks, out, scale);
    else readout_kernel<float><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, chunk0, nchunks, out, scale);
    return cudaGetLastError();
}

cudaError_t launch_block_mass(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B,
                              int C, CodecParams p, uint32_t nblocks, double *prefix, double *block_mass,
                              cudaStream_t s) {
    const unsigned grid = grid_for(nblocks, kPassThreads / 32, 8);
    if (f64)
        block_mass_kernel<double><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, nblocks, prefix,
                                                                block_mass);
    else
        block_mass_kernel<float><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, nblocks, prefix,
                                                               block_mass);
    return cudaGetLastError();
}

cudaError_t launch_sample_in_block(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask,
                                   int B, int C, CodecParams p, const double *prefix, const double *block_mass,
                                   const uint32_t *shot_block, const double *rin, uint64_t nshots, uint64_t *out,
                                   cudaStream_t s) {
    if (!nshots) return cudaSuccess;
    const unsigned grid = grid_for(nshots, kPassThreads / 32, 8);
    if (f64)
        sample_in_block_kernel<double><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, prefix,
                                                                     block_mass, shot_block, rin, nshots, out);
    else
        sample_in_block_kernel<float><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, prefix, block_mass,
                                                                    shot_block, rin, nshots, out);
    return cudaGetLastError();
}

cudaError_t launch_norm(bool f64, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *mask, int B, int C,
                        CodecParams p, uint64_t nchunks, double *out, cudaStream_t s) {
    const unsigned grid = grid_for(nchunks, kPassThreads / 32, 8);
    if (f64) norm_kernel<double><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, nchunks, out);
    else norm_kernel<float><<<grid, kPassThreads, 0, s>>>(meta, arena, mask, B, C, p, nchunks, out);
    return cudaGetLastError();
}

cudaError_t launch_encode(bool f64, const double *vals, int B, int C, CodecParams p, uint64_t chunk0, uint64_t nchunks,
                          ChunkMeta *meta, uint32_t *arena, unsigned long long *bump, uint64_t capacity,
                          uint32_t *block_nz, unsigned long long *block_bytes, int32_t *error, cudaStream_t s) {
    const unsigned grid = grid_for(nchunks, kPassThreads / 32, 8);
    if (f64)
        encode_kernel<double><<<grid, kPassThreads, 0, s>>>(vals, B, C, p, chunk0, nchunks, meta, arena, bump,
                                                           capacity, block_nz, block_bytes, error);
    else
        encode_kernel<float><<<grid, kPassThreads, 0, s>>>(vals, B, C, p, chunk0, nchunks, meta, arena, bump, capacity,
                                                          block_nz, block_bytes, error);
    return cudaGetLastError();
}

cudaError_t launch_codec_test(bool f64, const void *vals, int C, CodecParams p, uint64_t nchunks, uint32_t *words,
                              int32_t *bases, uint32_t *widths, void *decoded, cudaStream_t s) {
    const unsigned grid = grid_for(nchunks, kPassThreads / 32, 8);
    if (f64)
        codec_test_kernel<double><<<grid, kPassThreads, 0, s>>>((const double *)vals, C, p, nchunks, words, bases,
                                                               widths, (double *)decoded);
    else
        codec_test_kernel<float><<<grid, kPassThreads, 0, s>>>((const float *)vals, C, p, nchunks, words, bases, widths,
                                                              (float *)decoded);
    return cudaGetLastError();
}

uint64_t noalloc_scratch_words() { return kNoAllocScratchWords; }

template <typename R, int kC, int kJ>
static cudaError_t launch_dual_kc(const DualPassArgs &a, cudaStream_t s) {
    if (a.nslots > kMaxDualSlots) return cudaErrorInvalidValue;
    if (a.nsweeps > 0 && (a.rb != (sizeof(R) == 8 ? kDualRegBitsF64 : kDualRegBitsF32) || a.C + a.j < a.rb ||
                          a.nouter < 0 || a.nouter > kMaxOuterSel || !a.sweeps || !a.rops || !a.pool))
        return cudaErrorInvalidValue;
    const size_t smem = dual_pass_smem_bytes(sizeof(R) == 8, a.C, a.j);
    cudaError_t e = ensure_dyn_smem(dual_pass_kernel<R, kC, kJ>, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    const int threads = dual_threads(a.C + a.j);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dual_pass_kernel<R, kC, kJ>, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid == 0) grid = 1;
    dual_pass_kernel<R, kC, kJ><<<(unsigned)grid, threads, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_dual_t(const DualPassArgs &a, cudaStream_t s) {
    if (a.C == kMaxChunkLog2 && a.j == 4) return launch_dual_kc<R, kMaxChunkLog2, 4>(a, s);
    return launch_dual_kc<R, 0, 0>(a, s);
}

cudaError_t launch_dual_pass(bool f64, const DualPassArgs &a, cudaStream_t s) {
    return f64 ? launch_dual_t<double>(a, s) : launch_dual_t<float>(a, s);
}

cudaError_t launch_zero_unstored_headers(ChunkMeta *meta, const uint8_t *mask, uint64_t nchunks, int cshift,
                                         cudaStream_t s) {
    const unsigned grid = grid_for(nchunks, 256, 8);
    zero_unstored_headers_kernel<<<grid, 256, 0, s>>>(meta, mask, nchunks, cshift);
    return cudaGetLastError();
}

cudaError_t launch_half_sizes(const HalfChunks &h, const ChunkMeta *meta, const uint8_t *mask, uint64_t *sizes,
                              uint8_t *flags, cudaStream_t s) {
    if (h.nhalf == 0) return cudaSuccess;
    half_sizes_kernel<<<grid_for(h.nhalf, 256, 8), 256, 0, s>>>(h, meta, mask, sizes, flags);
    return cudaGetLastError();
}

uint64_t half_scan_scratch_words(uint64_t n) { return (n + kScanPerBlock - 1) / kScanPerBlock + 1; }

cudaError_t launch_half_scan(uint64_t *sizes, uint64_t n, uint64_t *scratch, uint64_t *total, cudaStream_t s) {
    const uint64_t m = (n + kScanPerBlock - 1) / kScanPerBlock;
    if (m == 0) return cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
    half_scan_blocks_kernel<<<(unsigned)m, kScanThreads, 0, s>>>(sizes, n, scratch);
    half_scan_totals_kernel<<<1, kScanThreads, 0, s>>>(scratch, m, total);
    half_scan_add_kernel<<<grid_for(n, 256, 8), 256, 0, s>>>(sizes, n, scratch);
    return cudaGetLastError();
}

cudaError_t launch_half_pack(const HalfChunks &h, const ChunkMeta *meta, const uint32_t *arena, const uint8_t *flags,
                             const uint64_t *offsets, ChunkMeta *out_meta, uint32_t *out_payload, bool scatter,
                             cudaStream_t s) {
    if (h.nhalf == 0) return cudaSuccess;
    half_pack_kernel<<<grid_for(h.nhalf * 32, 256, 8), 256, 0, s>>>(h, meta, arena, flags, offsets, out_meta,
                                                                    out_payload, scatter);
    return cudaGetLastError();
}

cudaError_t launch_half_unpack(const HalfChunks &h, const ChunkMeta *in_meta, const uint8_t *in_flags, uint64_t base,
                               ChunkMeta *meta, uint8_t *mask, cudaStream_t s) {
    if (h.nhalf == 0) return cudaSuccess;
    half_unpack_kernel<<<grid_for(h.nhalf, 256, 8), 256, 0, s>>>(h, in_meta, in_flags, base, meta, mask);
    return cudaGetLastError();
}

cudaError_t launch_half_check(const HalfChunks &h, const ChunkMeta *in_meta, const uint8_t *in_flags,
                              uint64_t payload_bytes_total, int32_t *bad, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(int32_t), s);
    if (e != cudaSuccess || h.nhalf == 0) return e;
    half_check_kernel<<<grid_for(h.nhalf, 256, 8), 256, 0, s>>>(h, in_meta, in_flags, payload_bytes_total, bad);
    return cudaGetLastError();
}

cudaError_t launch_bounded_wait_selftest(uint32_t tries, int32_t *gave_up, cudaStream_t s) {
    bounded_wait_selftest_kernel<<<1, 32, 0, s>>>(tries, gave_up);
    return cudaGetLastError();
}

cudaError_t launch_block_bytes(const ChunkMeta *meta, const uint8_t *mask, uint32_t nb, int cshift, int C,
                               unsigned long long *block_bytes, cudaStream_t s) {
    if (nb == 0) return cudaSuccess;
    block_bytes_kernel<<<grid_for((uint64_t)nb * 32, 256, 8), 256, 0, s>>>(meta, mask, nb, cshift, C, block_bytes);
    return cudaGetLastError();
}

template <typename R, int kC, int kJ>
static cudaError_t launch_adjoint_pass_kc(const AdjPassArgs &a, cudaStream_t s) {
    const int nb = a.C + a.j;
    const size_t smem = (size_t)(4 * sizeof(R)) << nb;
    auto kern = adjoint_pass_kernel<R, kC, kJ>;
    cudaError_t e = ensure_dyn_smem(kern, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kAdjThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid == 0) grid = 1;
    kern<<<(unsigned)grid, kAdjThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// The uncompressed adjoint's default geometry: 2^5-amplitude chunks and
// tiles of 2^11 (complex128) or 2^12 (complex64) amplitudes.
template <typename R>
static cudaError_t launch_adjoint_pass_t(const AdjPassArgs &a, cudaStream_t s) {
    if (a.nslots > kMaxAdjSlots) return cudaErrorInvalidValue;
    if (a.nsweeps > 0 && (a.rb != (sizeof(R) == 8 ? kDualRegBitsF64 : kDualRegBitsF32) || a.C + a.j < a.rb ||
                          a.nouter < 0 || a.nouter > kMaxOuterSel || !a.sweeps || !a.rops || !a.pool))
        return cudaErrorInvalidValue;
    constexpr int kAC = 5, kAJ = sizeof(R) == 8 ? 6 : 7;
    if (a.C == kAC && a.j == kAJ) return launch_adjoint_pass_kc<R, kAC, kAJ>(a, s);
    return launch_adjoint_pass_kc<R, 0, 0>(a, s);
}

cudaError_t launch_adjoint_pass(bool f64, const AdjPassArgs &a, cudaStream_t s) {
    return f64 ? launch_adjoint_pass_t<double>(a, s) : launch_adjoint_pass_t<float>(a, s);
}

// Host code may not use g_noalloc_words directly: in host code the name is a
// host-side stand-in, not a device address.  The device address is looked up
// with the device current on every call made outside a stream capture (a
// host-side table lookup once the module is loaded), so a device reset or a
// different context on the same device is picked up; a call inside a
// capture uses the address that the last call outside one found on that
// device (the first call on a device must come before any capture).
cudaError_t launch_codec_roundtrip_noalloc(bool f64, const void *vals, int C, CodecParams p, uint64_t nchunks,
                                           int32_t *bases, uint32_t *widths, void *decoded, cudaStream_t s) {
    static std::mutex mu;
    static void *addr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return e;
    uint32_t *words = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (cap == cudaStreamCaptureStatusNone || addr[dev] == nullptr) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_words);
            if (e != cudaSuccess) return e;
            addr[dev] = ptr;
        }
        words = static_cast<uint32_t *>(addr[dev]);
    }
    const unsigned grid = grid_for(nchunks, kPassThreads / 32, 8);
    if (f64)
        codec_test_kernel<double><<<grid, kPassThreads, 0, s>>>((const double *)vals, C, p, nchunks, words, bases,
                                                               widths, (double *)decoded);
    else
        codec_test_kernel<float><<<grid, kPassThreads, 0, s>>>((const float *)vals, C, p, nchunks, words, bases, widths,
                                                              (float *)decoded);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_expect_t(const ExpectArgs &a, cudaStream_t s) {
    if (a.nterms > kMaxTermsPerLaunch) return cudaErrorInvalidValue;
    const int nb = a.C + a.j;
    const size_t tiles = a.meta_bra ? 2 : 1;
    const size_t smem = tiles * ((size_t)(2 * sizeof(R)) << nb) + (size_t)(kExpectThreads / 32) * kStageWords * 4;
    cudaError_t e = ensure_dyn_smem(expect_kernel<R>, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, expect_kernel<R>, kExpectThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid == 0) grid = 1;
    expect_kernel<R><<<(unsigned)grid, kExpectThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_expect(bool f64, const ExpectArgs &a, cudaStream_t s) {
    return f64 ? launch_expect_t<double>(a, s) : launch_expect_t<float>(a, s);
}

cudaError_t launch_dense_expect(bool f64, const void *state, int n, const PauliTerm *terms, int nterms, double *out,
                                cudaStream_t s) {
    if (nterms > kMaxTermsPerLaunch) return cudaErrorInvalidValue;
    const unsigned grid = grid_for(uint64_t(1) << n, kExpectThreads, 8);
    if (f64)
        dense_expect_kernel<double><<<grid, kExpectThreads, 0, s>>>((const double2 *)state, (const double2 *)state, n,
                                                                   terms, nterms, out);
    else
        dense_expect_kernel<float><<<grid, kExpectThreads, 0, s>>>((const float2 *)state, (const float2 *)state, n, terms,
                                                                  nterms, out);
    return cudaGetLastError();
}

cudaError_t launch_dense_transition(bool f64, const void *bra, const void *ket, int n, const PauliTerm *terms,
                                    int nterms, double *out, cudaStream_t s) {
    if (nterms > kMaxTermsPerLaunch) return cudaErrorInvalidValue;
    const unsigned grid = grid_for(uint64_t(1) << n, kExpectThreads, 8);
    if (f64)
        dense_expect_kernel<double><<<grid, kExpectThreads, 0, s>>>((const double2 *)bra, (const double2 *)ket, n, terms,
                                                                   nterms, out);
    else
        dense_expect_kernel<float><<<grid, kExpectThreads, 0, s>>>((const float2 *)bra, (const float2 *)ket, n, terms,
                                                                  nterms, out);
    return cudaGetLastError();
}

template <typename R>
__global__ void dense_pauli_sum_kernel(const typename Cplx<R>::T *__restrict__ in, typename Cplx<R>::T *__restrict__ out,
                                       int n, const PauliTerm *__restrict__ terms, const double *__restrict__ coefs,
                                       int nterms) {
    using T = typename Cplx<R>::T;
    const uint64_t dim = uint64_t(1) << n;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int t = 0; t < nterms; ++t) {
            const uint64_t y = x ^ terms[t].xg;
            const T v = in[y];
            double cr = coefs[2 * t], ci = coefs[2 * t + 1];
            if (__popcll(y & terms[t].zg) & 1) { cr = -cr; ci = -ci; }
            re += cr * (double)v.x - ci * (double)v.y;
            im += cr * (double)v.y + ci * (double)v.x;
        }
        T o;
        o.x = (R)re;
        o.y = (R)im;
        out[x] = o;
    }
}

cudaError_t launch_dense_pauli_sum(bool f64, const void *in, void *out, int n, const PauliTerm *terms,
                                   const double *coefs, int nterms, cudaStream_t s) {
    const unsigned grid = grid_for(uint64_t(1) << n, 256, 8);
    if (f64)
        dense_pauli_sum_kernel<double><<<grid, 256, 0, s>>>((const double2 *)in, (double2 *)out, n, terms, coefs, nterms);
    else
        dense_pauli_sum_kernel<float><<<grid, 256, 0, s>>>((const float2 *)in, (float2 *)out, n, terms, coefs, nterms);
    return cudaGetLastError();
}

cudaError_t launch_dense_norm(bool f64, const void *state, uint64_t dim, double *out, cudaStream_t s) {
    const unsigned grid = grid_for(2 * dim, 256, 8);
    if (f64) dense_norm_kernel<double><<<grid, 256, 0, s>>>((const double *)state, 2 * dim, out);
    else dense_norm_kernel<float><<<grid, 256, 0, s>>>((const float *)state, 2 * dim, out);
    return cudaGetLastError();
}

cudaError_t launch_dense_to_c128(bool f64, const void *state, uint64_t dim, double *out, cudaStream_t s) {
    const unsigned grid = grid_for(2 * dim, 256, 8);
    if (f64) to_c128_kernel<double><<<grid, 256, 0, s>>>((const double *)state, 2 * dim, out);
    else to_c128_kernel<float><<<grid, 256, 0, s>>>((const float *)state, 2 * dim, out);
    return cudaGetLastError();
}

cudaError_t launch_c128_to_dense(bool f64, const double *in, uint64_t dim, void *state, cudaStream_t s) {
    const unsigned grid = grid_for(2 * dim, 256, 8);
    if (f64) from_c128_kernel<double><<<grid, 256, 0, s>>>(in, 2 * dim, (double *)state);
    else from_c128_kernel<float><<<grid, 256, 0, s>>>(in, 2 * dim, (float *)state);
    return cudaGetLastError();
}

}  // namespace qs
