// Host engine of the compressed state-vector path and the C ABI (qompsim.h).
//
// Restates the host logic of CompressedQuantumState
// (src/cppsim/compressed_state.hpp): block geometry and initial state
// (:87-239, :327-352), the stage partitioner partition_circuit (:509-583),
// make_block_groups (:585-671), partition_and_register_circuit (:673-726),
// register_circuit_stages (:464-507), the active-group rule of
// build_stage_group_execution_plan (:791-837), apply_circuit (:840-937),
// append_total_SV_bytes / get_max_SV_bytes (:374-445) and
// get_decompressed_state_vector (:1683-1707).
//
// What differs by design: the compressed store stays in device memory; a
// stage runs as one or more fused device passes (kernels.cu) instead of a
// host loop over groups with per-gate launches; the active-group test and
// the zero-mask update run on the device, so apply_circuit enqueues the
// whole circuit without a host synchronisation.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <unistd.h>

#include "../../include/qompsim.h"
#include "codec.cuh"
#include "internal.h"

using cplx = std::complex<double>;

namespace {

std::string g_last_error = "no error";

const char *kTimerKeys[10] = {"decomp", "gate", "comp", "fused_swap", "allgather",
                              "hmalloc", "dmalloc", "h2d", "d2h", "dfree"};

// --------------------------------------------------------------- gates
struct CGate {
    int nq = 0;
    int q[2] = {0, 0};
    cplx m[16];
    bool mix[2] = {false, false};
    bool diag = false;
};

// Express a matrix whose index bit i belongs to order[i] in ascending
// qubit order.
void reorder_ascending(int k, const int *order, const cplx *in, int *qout, cplx *out) {
    int idx[2] = {0, 1};
    if (k == 2 && order[0] > order[1]) std::swap(idx[0], idx[1]);
    for (int i = 0; i < k; ++i) qout[i] = order[idx[i]];
    const int dim = 1 << k;
    auto map = [&](int x) {  // new index -> old index
        int r = 0;
        for (int i = 0; i < k; ++i)
            if ((x >> i) & 1) r |= 1 << idx[i];
        return r;
    };
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) out[r * dim + c] = in[map(r) * dim + map(c)];
}

void compute_mixing(CGate *cg) {
    const int dim = 1 << cg->nq;
    for (int b = 0; b < cg->nq; ++b) {
        bool mx = false;
        for (int r = 0; r < dim; ++r)
            for (int c = 0; c < dim; ++c)
                if ((((r ^ c) >> b) & 1) && cg->m[r * dim + c] != cplx(0.0, 0.0)) mx = true;
        cg->mix[b] = mx;
    }
    if (cg->nq == 1) cg->mix[1] = false;
    cg->diag = !cg->mix[0] && !(cg->nq == 2 && cg->mix[1]);
}

bool canonicalize(const qs_gate &g, bool ref_controls, uint32_t n, CGate *cg, std::string *err) {
    const std::string name(g.name, strnlen(g.name, sizeof(g.name)));
    if (name == "FusedSWAP") {
        *err = "FusedSWAP gates exchange qubits between MPI ranks; this engine has one GPU and no ranks";
        return false;
    }
    if (g.ntargets < 1 || g.ntargets > 2 || g.ncontrols > 2) {
        *err = "Error: only single- or two-qubit gates are implemented";
        return false;
    }
    for (uint32_t i = 0; i < g.ntargets; ++i)
        if (g.targets[i] >= n) { *err = "gate target index out of range"; return false; }
    for (uint32_t i = 0; i < g.ncontrols; ++i)
        if (g.controls[i] >= n) { *err = "gate control index out of range"; return false; }
    const int nt = (int)g.ntargets;
    const int dimt = 1 << nt;
    cplx M[16];
    for (int k = 0; k < dimt * dimt; ++k) M[k] = cplx(g.matrix[2 * k], g.matrix[2 * k + 1]);
    const bool use_controls = !ref_controls || name == "CNOT";
    if (use_controls && g.ncontrols > 0) {
        const int k = nt + (int)g.ncontrols;
        if (k > 2) {
            *err = "Error: only single- or two-qubit gates are implemented (targets + controls > 2)";
            return false;
        }
        int order[2];
        for (int i = 0; i < nt; ++i) order[i] = (int)g.targets[i];
        for (int i = 0; i < (int)g.ncontrols; ++i) order[nt + i] = (int)g.controls[i];
        if (order[0] == order[1]) { *err = "duplicated qubit index in gate"; return false; }
        cplx F[16];
        const int dim = 1 << k;
        for (int r = 0; r < dim; ++r)
            for (int c = 0; c < dim; ++c) F[r * dim + c] = r == c ? 1.0 : 0.0;
        int cm = 0;
        for (int i = 0; i < (int)g.ncontrols; ++i)
            if (g.control_values[i]) cm |= 1 << i;
        const int base = cm << nt;
        for (int r = 0; r < dimt; ++r)
            for (int c = 0; c < dimt; ++c) F[(base + r) * dim + base + c] = M[r * dimt + c];
        cg->nq = k;
        reorder_ascending(k, order, F, cg->q, cg->m);
    } else if (nt == 1) {
        cg->nq = 1;
        cg->q[0] = (int)g.targets[0];
        for (int k2 = 0; k2 < 4; ++k2) cg->m[k2] = M[k2];
    } else {
        if (g.targets[0] == g.targets[1]) { *err = "duplicated qubit index in gate"; return false; }
        cg->nq = 2;
        if (ref_controls) {
            // The reference's two-qubit kernels pair matrix bit 0 with the lower
            // target whatever the target order (compressed_state_cuda.cu:632-642).
            cg->q[0] = (int)std::min(g.targets[0], g.targets[1]);
            cg->q[1] = (int)std::max(g.targets[0], g.targets[1]);
            for (int k2 = 0; k2 < 16; ++k2) cg->m[k2] = M[k2];
        } else {
            int order[2] = {(int)g.targets[0], (int)g.targets[1]};
            reorder_ascending(2, order, M, cg->q, cg->m);
        }
    }
    compute_mixing(cg);
    return true;
}

// A gate whose qubits are all >= C and whose matrix sends every basis state
// to one basis state with coefficient exactly 1 by moving and flipping bits
// (I, X, SWAP and their products): it permutes whole chunks.  *swap: the
// gate exchanges its two qubits; *flip: matrix bits flipped after that.
bool chunk_perm_gate(const CGate &g, int C, bool *swap, int *flip) {
    for (int i = 0; i < g.nq; ++i)
        if (g.q[i] < C) return false;
    const int dim = 1 << g.nq;
    int f[4];
    for (int c = 0; c < dim; ++c) {
        f[c] = -1;
        for (int r = 0; r < dim; ++r) {
            const cplx v = g.m[r * dim + c];
            if (v == cplx(1.0, 0.0)) {
                if (f[c] >= 0) return false;
                f[c] = r;
            } else if (v != cplx(0.0, 0.0)) {
                return false;
            }
        }
        if (f[c] < 0) return false;
    }
    const int x = f[0];
    *flip = x;
    if (g.nq == 1) {
        *swap = false;
        return f[1] == (1 ^ x);
    }
    if ((f[1] ^ x) == 1 && (f[2] ^ x) == 2 && (f[3] ^ x) == 3) {
        *swap = false;
        return true;
    }
    if ((f[1] ^ x) == 2 && (f[2] ^ x) == 1 && (f[3] ^ x) == 3) {
        *swap = true;
        return true;
    }
    return false;
}

// Chunk-index permutation sigma(c) = pi(c) ^ x accumulated over the SWAP / X
// gates of a stage (bits are qubit - C).  The stage's true state is
// psi_true[sigma(i)] = psi_stored[i]; a later gate G is applied to the stored
// state as sigma^-1 G sigma (relabel()), and the last pass of the stage
// writes chunk c to position sigma(c).
struct HostPerm {
    std::vector<int> dst;  // dst[s] = pi(s)
    uint64_t x = 0;
    explicit HostPerm(int bits) : dst(bits) {
        for (int s = 0; s < bits; ++s) dst[s] = s;
    }
    bool identity() const {
        if (x) return false;
        for (size_t s = 0; s < dst.size(); ++s)
            if (dst[s] != (int)s) return false;
        return true;
    }
    void then_swap(int a, int b) {
        for (auto &d : dst) {
            if (d == a) d = b;
            else if (d == b) d = a;
        }
        const uint64_t ba = (x >> a) & 1, bb = (x >> b) & 1;
        x &= ~((1ull << a) | (1ull << b));
        x |= (ba << b) | (bb << a);
    }
    void then_flip(int a) { x ^= 1ull << a; }
    int inverse(int q) const {
        for (size_t s = 0; s < dst.size(); ++s)
            if (dst[s] == q) return (int)s;
        return q;
    }
    qs::ChunkPerm device() const {
        qs::ChunkPerm p;
        std::memset(&p, 0, sizeof(p));
        p.keep = ~0ull;
        p.flip = x;
        for (size_t s = 0; s < dst.size(); ++s) {
            if (dst[s] == (int)s) continue;
            p.keep &= ~(1ull << s);
            p.src[p.nmove] = (int8_t)s;
            p.dst[p.nmove] = (int8_t)dst[s];
            ++p.nmove;
        }
        return p;
    }
};

CGate relabel(const CGate &g, const HostPerm &P, int C);

// The gates of one stage as the device applies them: SWAP / X gates on
// qubits >= C are folded into P (when enabled) and every other gate is
// relabelled through the permutation accumulated before it.
void stage_relabel(const std::vector<CGate> &cgates, const std::vector<uint32_t> &ids, int C, bool enable,
                   std::vector<CGate> *out, HostPerm *P) {
    out->clear();
    for (uint32_t gi : ids) {
        const CGate &g = cgates[gi];
        bool sw = false;
        int fl = 0;
        if (enable && chunk_perm_gate(g, C, &sw, &fl)) {
            // the gate acts after the permutation so far: sigma <- gate o sigma
            if (sw) P->then_swap(g.q[0] - C, g.q[1] - C);
            for (int i = 0; i < g.nq; ++i)
                if ((fl >> i) & 1) P->then_flip(g.q[i] - C);
            continue;
        }
        out->push_back(relabel(g, *P, C));
    }
}

qs::ChunkPerm identity_perm() {
    qs::ChunkPerm p;
    std::memset(&p, 0, sizeof(p));
    p.keep = ~0ull;
    return p;
}

// sigma^-1 G sigma: G on qubit q >= C acts on stored qubit pi^-1(q - C) + C,
// with the matrix index bit flipped where x has bit q - C.
CGate relabel(const CGate &g, const HostPerm &P, int C) {
    CGate o = g;
    int F = 0;
    int order[2] = {g.q[0], g.q[1]};
    for (int i = 0; i < g.nq; ++i) {
        if (g.q[i] < C) continue;
        const int b = g.q[i] - C;
        order[i] = P.inverse(b) + C;
        if ((P.x >> b) & 1) F |= 1 << i;
    }
    const int dim = 1 << g.nq;
    cplx M[16];
    for (int r = 0; r < dim; ++r)
        for (int c = 0; c < dim; ++c) M[r * dim + c] = g.m[(r ^ F) * dim + (c ^ F)];
    if (g.nq == 2) {
        reorder_ascending(2, order, M, o.q, o.m);
    } else {
        o.q[0] = order[0];
        for (int k = 0; k < 4; ++k) o.m[k] = M[k];
    }
    compute_mixing(&o);
    return o;
}

qs::KGate to_kgate(const CGate &cg, const std::vector<int> &tile_qubits, int C) {
    qs::KGate k;
    std::memset(&k, 0, sizeof(k));
    k.nq = cg.nq;
    k.diag = cg.diag ? 1 : 0;
    k.mixmask = (cg.mix[0] ? 1 : 0) | (cg.nq == 2 && cg.mix[1] ? 2 : 0);
    for (int i = 0; i < cg.nq; ++i) {
        k.q[i] = cg.q[i];
        if (cg.q[i] < C) {
            k.tpos[i] = cg.q[i];
        } else {
            auto it = std::find(tile_qubits.begin(), tile_qubits.end(), cg.q[i]);
            k.tpos[i] = it == tile_qubits.end() ? -1 : C + (int)(it - tile_qubits.begin());
        }
    }
    const int dim = 1 << cg.nq;
    for (int r = 0; r < dim * dim; ++r) {
        k.m[2 * r] = cg.m[r].real();
        k.m[2 * r + 1] = cg.m[r].imag();
    }
    return k;
}

// Group the gates [g0, g1) of a pass (already in KGate form) into register
// sweeps: consecutive gates whose mixing tile bits fit in RB bits share a
// sweep; the sweep's bit set is padded with the lowest free tile bits.
std::vector<qs::Sweep> plan_sweeps(const std::vector<qs::KGate> &kg, size_t g0, size_t g1, int nb, int RB) {
    std::vector<qs::Sweep> out;
    std::set<int> S;
    size_t start = g0;
    auto close = [&](size_t end) {
        qs::Sweep sw{};
        sw.g0 = (int32_t)(start - g0);
        sw.g1 = (int32_t)(end - g0);
        for (int b = 0; b < nb && (int)S.size() < RB; ++b) S.insert(b);
        int k = 0;
        for (int b : S) sw.sbits[k++] = b;
        out.push_back(sw);
        S.clear();
        start = end;
    };
    for (size_t i = g0; i < g1; ++i) {
        std::set<int> need = S;
        for (int b = 0; b < kg[i].nq; ++b)
            if ((kg[i].mixmask >> b) & 1) need.insert(kg[i].tpos[b]);
        if ((int)need.size() > RB) {
            close(i);
            for (int b = 0; b < kg[i].nq; ++b)
                if ((kg[i].mixmask >> b) & 1) S.insert(kg[i].tpos[b]);
        } else {
            S = need;
        }
    }
    if (g1 > start || out.empty()) close(g1);
    return out;
}

// Resolve the gates [g0, g1) of a pass against their sweeps into op records
// and sub-matrix variants (appended to *ops and *pool).  Sweep gate ranges are
// relative to g0; op k of the pass is gate g0 + k.
// A register op before its final encoding: kind, register bits, selector
// sources (< 64: tile bit, >= 64: outer qubit + 64) and its variants in the
// pool (variant v at mat + v * vstride).
// RK_SUM (two-store sweeps): a derivative sum, xs / zs its register masks,
// slot its local slot, one +-1 sign per variant (vstride 1).
enum RawKind : uint8_t { RK_SCALAR = 0, RK_D2 = 1, RK_M2 = 2, RK_D4 = 3, RK_M4 = 4, RK_SUM = 5 };
struct RawOp {
    uint8_t kind = RK_SCALAR;
    uint8_t k0 = 0, k1 = 0;
    uint8_t nsel = 0;
    uint8_t sel[qs::kMaxSel] = {};
    uint32_t mat = 0, vstride = 0;
    uint8_t xs = 0, zs = 0;
    int32_t slot = -1;
};

void build_gate_op(const qs::KGate &g, const qs::Sweep &sw, int RB, std::vector<RawOp> *ops, std::vector<cplx> *pool);

void build_ops(const std::vector<qs::KGate> &kg, size_t g0, const std::vector<qs::Sweep> &sweeps, int RB,
               std::vector<RawOp> *ops, std::vector<cplx> *pool) {
    for (const auto &sw : sweeps)
        for (int gi = sw.g0; gi < sw.g1; ++gi) build_gate_op(kg[g0 + gi], sw, RB, ops, pool);
}

// The derivative sum of a gate whose generator has flip mask gx and Z mask gz
// (global qubits), as a register op of sweep sw: flips must lie on register
// bits; Z factors on other qubits select a +-1 variant.  tile: the pass's
// tile qubits >= C.  False when a flip qubit is not a register bit.
bool build_sum_op(uint64_t gx, uint64_t gz, int slot, const qs::Sweep &sw, int RB, const std::vector<int> &tile, int C,
                  std::vector<RawOp> *ops, std::vector<cplx> *pool) {
    RawOp op{};
    op.kind = RK_SUM;
    op.slot = slot;
    op.vstride = 1;
    for (int q = 0; q < 64; ++q) {
        const bool xb = (gx >> q) & 1, zb = (gz >> q) & 1;
        if (!xb && !zb) continue;
        int p = q < C ? q : -1;
        if (q >= C) {
            auto it = std::find(tile.begin(), tile.end(), q);
            if (it != tile.end()) p = C + (int)(it - tile.begin());
        }
        int k = -1;
        for (int kk = 0; kk < RB; ++kk)
            if (p >= 0 && sw.sbits[kk] == p) k = kk;
        if (k >= 0) {
            op.xs |= (uint8_t)(xb << k);
            op.zs |= (uint8_t)(zb << k);
        } else {
            if (xb || op.nsel >= qs::kMaxSel) return false;
            op.sel[op.nsel++] = (uint8_t)(p >= 0 ? p : 64 + q);
        }
    }
    op.mat = (uint32_t)pool->size();
    for (int v = 0; v < (1 << op.nsel); ++v) pool->push_back(cplx((__builtin_popcount(v) & 1) ? -1.0 : 1.0, 0.0));
    ops->push_back(op);
    return true;
}

void build_gate_op(const qs::KGate &g, const qs::Sweep &sw, int RB, std::vector<RawOp> *ops, std::vector<cplx> *pool) {
    int reg[2] = {-1, -1}, src[2] = {0, 0};
    std::vector<int> fixed;  // gate-qubit indices that select a variant
    for (int i = 0; i < g.nq; ++i) {
        const int p = g.tpos[i];
        int k = -1;
        for (int kk = 0; kk < RB; ++kk)
            if (p >= 0 && sw.sbits[kk] == p) k = kk;
        if (k >= 0) {
            reg[i] = k;
        } else {
            src[i] = p >= 0 ? p : 64 + g.q[i];
            fixed.push_back(i);
        }
    }
    const int dim = 1 << g.nq;
    auto M = [&](int r, int c) { return cplx(g.m[2 * (r * dim + c)], g.m[2 * (r * dim + c) + 1]); };
    std::vector<int> regs;
    for (int i = 0; i < g.nq; ++i)
        if (reg[i] >= 0) regs.push_back(i);
    RawOp op{};
    op.nsel = (uint8_t)fixed.size();
    for (size_t j = 0; j < fixed.size(); ++j) op.sel[j] = (uint8_t)src[fixed[j]];
    op.mat = (uint32_t)pool->size();
    const int nvar = 1 << fixed.size();
    // full-matrix index of register pattern x under variant v
    auto full = [&](int x, int v) {
        int idx = 0;
        for (size_t r = 0; r < regs.size(); ++r)
            if ((x >> r) & 1) idx |= 1 << regs[r];
        for (size_t j = 0; j < fixed.size(); ++j)
            if ((v >> j) & 1) idx |= 1 << fixed[j];
        return idx;
    };
    const int rd = 1 << regs.size();
    bool diag = true;
    for (int v = 0; v < nvar; ++v)
        for (int x = 0; x < rd; ++x)
            for (int y = 0; y < rd; ++y)
                if (x != y && M(full(x, v), full(y, v)) != cplx(0, 0)) diag = false;
    if (regs.empty()) {
        op.kind = RK_SCALAR;
        op.vstride = 1;
        for (int v = 0; v < nvar; ++v) pool->push_back(M(full(0, v), full(0, v)));
    } else if (regs.size() == 1) {
        op.k0 = (uint8_t)reg[regs[0]];
        if (diag) {
            op.kind = RK_D2;
            op.vstride = 2;
            for (int v = 0; v < nvar; ++v) {
                pool->push_back(M(full(0, v), full(0, v)));
                pool->push_back(M(full(1, v), full(1, v)));
            }
        } else {
            op.kind = RK_M2;
            op.vstride = 4;
            for (int v = 0; v < nvar; ++v)
                for (int x = 0; x < 2; ++x)
                    for (int y = 0; y < 2; ++y) pool->push_back(M(full(x, v), full(y, v)));
        }
    } else {
        op.k0 = (uint8_t)reg[0];
        op.k1 = (uint8_t)reg[1];
        if (diag) {
            op.kind = RK_D4;
            op.vstride = 4;
            for (int x = 0; x < 4; ++x) pool->push_back(M(x, x));
        } else {
            op.kind = RK_M4;
            op.vstride = 16;
            for (int x = 0; x < 16; ++x) pool->push_back(M(x / 4, x % 4));
        }
    }
    ops->push_back(op);
}

// Merge runs of diagonal ops: a SCALAR or D2 op followed by SCALAR / D2 ops
// on the same register bit becomes one D2 (or SCALAR) op whose variants
// range over the union of the selector bits (at most kMaxSel).  The merged
// op's variant v multiplies the factors of every member at its own variant
// (v restricted to the member's selector bits).  Applied per sweep.
void merge_diagonal_ops(const std::vector<qs::Sweep> &sweeps, size_t op0, std::vector<RawOp> *ops,
                        std::vector<cplx> *pool, std::vector<qs::Sweep> *out_sweeps) {
    std::vector<RawOp> out;
    std::vector<cplx> outpool;
    out_sweeps->clear();
    for (const auto &sw : sweeps) {
        qs::Sweep ns = sw;
        ns.g0 = (int32_t)out.size();
        size_t i = op0 + sw.g0;
        const size_t end = op0 + sw.g1;
        while (i < end) {
            const RawOp &a = (*ops)[i];
            auto is_diag1 = [](const RawOp &o) { return o.kind == RK_SCALAR || o.kind == RK_D2; };
            if (!is_diag1(a)) {
                RawOp c = a;
                c.mat = (uint32_t)outpool.size();
                const int nvar = 1 << a.nsel;
                for (int v = 0; v < nvar; ++v)
                    for (uint32_t e = 0; e < a.vstride; ++e) outpool.push_back((*pool)[a.mat + v * a.vstride + e]);
                out.push_back(c);
                ++i;
                continue;
            }
            // grow a run [i, j) of diagonal ops on one register bit (or scalars)
            int k = a.kind == RK_D2 ? a.k0 : -1;
            std::vector<int> sels(a.sel, a.sel + a.nsel);
            size_t j = i + 1;
            while (j < end && is_diag1((*ops)[j])) {
                const RawOp &b = (*ops)[j];
                if (b.kind == RK_D2 && k >= 0 && b.k0 != k) break;
                std::vector<int> u = sels;
                for (int t = 0; t < b.nsel; ++t)
                    if (std::find(u.begin(), u.end(), (int)b.sel[t]) == u.end()) u.push_back(b.sel[t]);
                if ((int)u.size() > qs::kMaxSel) break;
                sels = u;
                if (b.kind == RK_D2) k = b.k0;
                ++j;
            }
            RawOp m{};
            m.kind = k >= 0 ? RK_D2 : RK_SCALAR;
            m.k0 = (uint8_t)(k >= 0 ? k : 0);
            m.nsel = (uint8_t)sels.size();
            for (size_t t = 0; t < sels.size(); ++t) m.sel[t] = (uint8_t)sels[t];
            m.vstride = k >= 0 ? 2 : 1;
            m.mat = (uint32_t)outpool.size();
            const int nvar = 1 << sels.size();
            for (int v = 0; v < nvar; ++v) {
                cplx f0 = 1.0, f1 = 1.0;
                for (size_t t = i; t < j; ++t) {
                    const RawOp &b = (*ops)[t];
                    int bv = 0;
                    for (int q = 0; q < b.nsel; ++q) {
                        const int pos = (int)(std::find(sels.begin(), sels.end(), (int)b.sel[q]) - sels.begin());
                        bv |= ((v >> pos) & 1) << q;
                    }
                    if (b.kind == RK_SCALAR) {
                        const cplx z = (*pool)[b.mat + bv];
                        f0 *= z;
                        f1 *= z;
                    } else {
                        f0 *= (*pool)[b.mat + 2 * bv];
                        f1 *= (*pool)[b.mat + 2 * bv + 1];
                    }
                }
                outpool.push_back(f0);
                if (k >= 0) outpool.push_back(f1);
            }
            out.push_back(m);
            i = j;
        }
        ns.g1 = (int32_t)out.size();
        out_sweeps->push_back(ns);
    }
    // replace this pass's ops [op0, ...) and pool suffix
    ops->resize(op0);
    const uint32_t pbase = (uint32_t)pool->size();
    for (auto &o : out) o.mat += pbase;
    ops->insert(ops->end(), out.begin(), out.end());
    pool->insert(pool->end(), outpool.begin(), outpool.end());
}

// Final encoding of one pass's raw ops (codes in internal.h): selector
// sources become bit positions of the group word W (tile bit p -> p, outer
// qubit q -> nb + its index in *outer), register bit pairs are put in
// ascending order, and the variants are laid out for the code.  Diagonals
// whose bit-0 factor is exactly 1 in every variant touch only the bit-1
// amplitudes; exact X and SWAP matrices become register moves.  Appends to
// ops/pool; false when the pass needs more than kMaxOuterSel outer qubits.
// When an op's selector bits form at most two runs of consecutive positions
// of W, its variants are renumbered so that variant bit j is the j-th
// selector in ascending position, and the op carries the runs instead of the
// bit list (sel[0] = kSelRuns | start1, sel[1] = length1, sel[2] = start2,
// sel[3] = length2): the device then computes the variant with two shifts
// and masks instead of one extract per selector.  stride: pool entries per
// variant, starting at o->mat (the op's entries are the last ones appended).
void encode_selector_runs(qs::ROp *o, int stride, std::vector<cplx> *pool) {
    const int ns = o->nsel;
    if (ns == 0 || stride == 0) return;
    std::vector<int> order(ns);
    for (int j = 0; j < ns; ++j) order[j] = j;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return o->sel[a] < o->sel[b]; });
    int runs = 1, start[2] = {o->sel[order[0]], 0}, len[2] = {1, 0};
    for (int j = 1; j < ns; ++j) {
        if (o->sel[order[j]] == o->sel[order[j - 1]] + 1) {
            ++len[runs - 1];
        } else {
            if (++runs > 2) return;
            start[1] = o->sel[order[j]];
            len[1] = 1;
        }
    }
    const size_t nvar = size_t(1) << ns;
    std::vector<cplx> old(pool->begin() + o->mat, pool->begin() + o->mat + nvar * stride);
    for (size_t vn = 0; vn < nvar; ++vn) {
        size_t vo = 0;
        for (int j = 0; j < ns; ++j)
            if ((vn >> j) & 1) vo |= size_t(1) << order[j];
        for (int e = 0; e < stride; ++e) (*pool)[o->mat + vn * stride + e] = old[vo * stride + e];
    }
    for (int j = 0; j < qs::kMaxSel; ++j) o->sel[j] = 0;
    o->sel[0] = (uint8_t)(qs::kSelRuns | start[0]);
    o->sel[1] = (uint8_t)len[0];
    o->sel[2] = (uint8_t)start[1];
    o->sel[3] = (uint8_t)len[1];
}

// Runs of half-diagonal ops on one register bit inside a sweep (phases that
// the diagonal merge could not join because their selectors are too many):
// every op but the last only multiplies a pending factor (OPC_ACC), the last
// (OPC_D2HP) applies the product once.  ops[op0 + sweep.g0 .. g1) per sweep.
void fuse_half_chains(std::vector<qs::ROp> *ops, size_t op0, const std::vector<qs::Sweep> &sweeps) {
    for (const auto &sw : sweeps)
        for (int k = sw.g0 + 1; k < sw.g1; ++k) {
            qs::ROp &prev = (*ops)[op0 + k - 1], &cur = (*ops)[op0 + k];
            if (cur.code < qs::OPC_D2H || cur.code >= qs::OPC_D2H + 8) continue;
            const int bit = cur.code - qs::OPC_D2H;
            const bool chained = prev.code == qs::OPC_D2H + bit || prev.code == qs::OPC_D2HP + bit;
            if (!chained) continue;
            prev.code = qs::OPC_ACC;
            cur.code = (uint8_t)(qs::OPC_D2HP + bit);
        }
}

bool finalize_ops(const std::vector<RawOp> &raw, const std::vector<cplx> &rpool, int nb, std::vector<int> *outer,
                  std::vector<qs::ROp> *ops, std::vector<cplx> *pool) {
    const cplx one(1.0, 0.0), zero(0.0, 0.0);
    for (const RawOp &r : raw) {
        qs::ROp o;
        std::memset(&o, 0, sizeof(o));
        o.nsel = r.nsel;
        for (int j = 0; j < qs::kMaxSel; ++j) o.sel[j] = qs::kSelNone;
        for (int j = 0; j < r.nsel; ++j) {
            const int src = r.sel[j];
            if (src < 64) {
                o.sel[j] = (uint8_t)src;
                continue;
            }
            auto it = std::find(outer->begin(), outer->end(), src - 64);
            if (it == outer->end()) {
                if ((int)outer->size() >= qs::kMaxOuterSel) return false;
                outer->push_back(src - 64);
                it = outer->end() - 1;
            }
            o.sel[j] = (uint8_t)(nb + (it - outer->begin()));
        }
        const int nvar = 1 << r.nsel;
        auto E = [&](int v, int e) { return rpool[r.mat + (size_t)v * r.vstride + e]; };
        o.mat = (uint32_t)pool->size();
        const int a = std::min(r.k0, r.k1), b = std::max(r.k0, r.k1);
        const bool flip = r.k0 > r.k1;  // canonical index: bit 0 <-> the lower register bit
        auto canon = [&](int x) { return flip ? (((x & 1) << 1) | (x >> 1)) : x; };
        switch (r.kind) {
            case RK_SUM:
                o.code = qs::OPC_SUM;
                o.vstride = (uint8_t)r.slot;
                o.pad = (uint8_t)((r.xs << 4) | r.zs);
                for (int v = 0; v < nvar; ++v) pool->push_back(E(v, 0));
                break;
            case RK_SCALAR:
                o.code = qs::OPC_SCALAR;
                o.vstride = 1;
                for (int v = 0; v < nvar; ++v) pool->push_back(E(v, 0));
                break;
            case RK_D2: {
                bool unit = true;
                for (int v = 0; v < nvar; ++v) unit = unit && E(v, 0) == one;
                o.code = (uint8_t)((unit ? qs::OPC_D2H : qs::OPC_D2) + r.k0);
                o.vstride = unit ? 1 : 2;
                for (int v = 0; v < nvar; ++v) {
                    if (!unit) pool->push_back(E(v, 0));
                    pool->push_back(E(v, 1));
                }
                break;
            }
            case RK_M2:
                if (r.nsel == 0 && E(0, 0) == zero && E(0, 1) == one && E(0, 2) == one && E(0, 3) == zero) {
                    o.code = (uint8_t)(qs::OPC_X + r.k0);
                    o.vstride = 0;
                } else {
                    o.code = (uint8_t)(qs::OPC_M2 + r.k0);
                    o.vstride = 4;
                    for (int v = 0; v < nvar; ++v)
                        for (int e = 0; e < 4; ++e) pool->push_back(E(v, e));
                }
                break;
            case RK_D4: {
                bool unit = true;
                for (int v = 0; v < nvar; ++v) unit = unit && E(v, canon(0)) == one;
                o.code = (uint8_t)((unit ? qs::OPC_D4H : qs::OPC_D4) + a * 8 + b);
                o.vstride = unit ? 3 : 4;
                for (int v = 0; v < nvar; ++v)
                    for (int y = unit ? 1 : 0; y < 4; ++y) pool->push_back(E(v, canon(y)));
                break;
            }
            default: {  // RK_M4
                std::vector<cplx> m(16 * (size_t)nvar);
                for (int v = 0; v < nvar; ++v)
                    for (int y = 0; y < 4; ++y)
                        for (int x = 0; x < 4; ++x) m[16 * v + 4 * y + x] = E(v, 4 * canon(y) + canon(x));
                bool is_swap = r.nsel == 0;
                for (int y = 0; y < 4 && is_swap; ++y)
                    for (int x = 0; x < 4; ++x) {
                        const int t = (y == 1) ? 2 : (y == 2) ? 1 : y;
                        if (m[4 * y + x] != (x == t ? one : zero)) is_swap = false;
                    }
                if (is_swap) {
                    o.code = (uint8_t)(qs::OPC_SWAP + a * 8 + b);
                    o.vstride = 0;
                } else {
                    o.code = (uint8_t)(qs::OPC_M4 + a * 8 + b);
                    o.vstride = 16;
                    pool->insert(pool->end(), m.begin(), m.end());
                }
                break;
            }
        }
        encode_selector_runs(&o, r.kind == RK_SUM ? 1 : o.vstride, pool);
        ops->push_back(o);
    }
    return true;
}

template <typename Real>
std::vector<Real> pool_as(const std::vector<cplx> &pool) {
    std::vector<Real> out(2 * pool.size());
    for (size_t i = 0; i < pool.size(); ++i) {
        out[2 * i] = (Real)pool[i].real();
        out[2 * i + 1] = (Real)pool[i].imag();
    }
    return out;
}

// Register sweeps over two stores for one launch of a backward pass: the
// gates `gl` (indices into cg) in order, the derivative sum of each
// parametric one (slots[gi] >= 0; local slots numbered in order) placed just
// before it as a pseudo-gate with the gate's qubits and mixing bits, so that
// the two share a sweep and the generator's flip qubits are register bits.
// Appends sweeps (op ranges relative to *rop_off), ops and variants; false
// (nothing appended) when a flip qubit is not a register bit or the pass
// needs too many outer selector qubits.
struct DualSweepPlan {
    size_t sw_off = 0, nsw = 0, rop_off = 0;
    std::vector<int> outer;
};
bool plan_dual_sweeps(const std::vector<CGate> &cg, const std::vector<uint32_t> &gl, const int32_t *slots,
                      const uint64_t *gen_x, const uint64_t *gen_z, const std::vector<int> &tile, int C, int RB,
                      std::vector<qs::Sweep> *all_sw, std::vector<qs::ROp> *all_rops, std::vector<cplx> *all_pool,
                      DualSweepPlan *out);

struct PassPlan {
    std::vector<int> tile;        // tile qubits >= C, ascending
    std::vector<uint32_t> gates;  // indices into the gate list
};

// Split a gate sequence into passes: a pass's tile holds the chunk qubits
// [0, C) plus at most jmax other qubits, which must include every qubit on
// which a gate of the pass mixes amplitudes.  Tiles are padded to jmin
// qubits with in-block qubits so that a tile has several chunks.
std::vector<PassPlan> plan_passes(const std::vector<uint32_t> &gate_ids, const std::vector<CGate> &cg, int C,
                                  int jmax, int jmin, int pad_lo, int pad_hi) {
    std::vector<PassPlan> out;
    std::set<int> cur, sel;  // mixing qubits >= C; non-mixing qubits >= C (selector candidates)
    PassPlan p;
    auto outside = [](const std::set<int> &a, const std::set<int> &t) {
        int k = 0;
        for (int q : a) k += t.count(q) ? 0 : 1;
        return k;
    };
    for (uint32_t gi : gate_ids) {
        std::set<int> need = cur, nsel = sel;
        for (int b = 0; b < cg[gi].nq; ++b) {
            if (cg[gi].q[b] < C) continue;
            (cg[gi].mix[b] ? need : nsel).insert(cg[gi].q[b]);
        }
        if ((int)need.size() > jmax || outside(nsel, need) > qs::kMaxOuterSel) {
            p.tile.assign(cur.begin(), cur.end());
            out.push_back(p);
            p = PassPlan();
            cur.clear();
            sel.clear();
            for (int b = 0; b < cg[gi].nq; ++b) {
                if (cg[gi].q[b] < C) continue;
                (cg[gi].mix[b] ? cur : sel).insert(cg[gi].q[b]);
            }
        } else {
            cur = need;
            sel = nsel;
        }
        p.gates.push_back(gi);
    }
    p.tile.assign(cur.begin(), cur.end());
    out.push_back(p);
    for (auto &pp : out) {
        std::set<int> s(pp.tile.begin(), pp.tile.end());
        for (int q = pad_lo; q < pad_hi && (int)s.size() < jmin; ++q) s.insert(q);
        pp.tile.assign(s.begin(), s.end());
    }
    return out;
}

// The same split with commuting gates reordered: two gates that share a
// qubit commute when neither mixes amplitudes along it (both are then
// block-diagonal in that qubit and act on disjoint other qubits), so a gate
// waits only for the earlier gates it does not commute with.  Each pass
// takes, in index order and repeatedly, every ready gate whose mixing qubits
// >= C still fit the tile and whose other qubits >= C fit the outer
// selectors; a gate made ready by one taken in this pass may join it.  A
// pass's gate list is a valid order of its gates.
std::vector<PassPlan> plan_passes_dag(const std::vector<uint32_t> &gate_ids, const std::vector<CGate> &cg, int C,
                                      int jmax, int jmin, int pad_lo, int pad_hi) {
    const size_t G = gate_ids.size();
    std::vector<std::vector<uint32_t>> succ(G);
    std::vector<int> indeg(G, 0);
    {
        std::vector<int> last_mix;                 // per qubit: last gate mixing it
        std::vector<std::vector<uint32_t>> users;  // per qubit: non-mixing gates since then
        for (size_t i = 0; i < G; ++i) {
            const CGate &g = cg[gate_ids[i]];
            std::vector<uint32_t> preds;
            for (int b = 0; b < g.nq; ++b) {
                const int q = g.q[b];
                if ((int)last_mix.size() <= q) {
                    last_mix.resize(q + 1, -1);
                    users.resize(q + 1);
                }
                if (last_mix[q] >= 0) preds.push_back((uint32_t)last_mix[q]);
                if (g.mix[b]) {
                    preds.insert(preds.end(), users[q].begin(), users[q].end());
                    last_mix[q] = (int)i;
                    users[q].clear();
                } else {
                    users[q].push_back((uint32_t)i);
                }
            }
            std::sort(preds.begin(), preds.end());
            preds.erase(std::unique(preds.begin(), preds.end()), preds.end());
            for (uint32_t p : preds) {
                succ[p].push_back((uint32_t)i);
                ++indeg[i];
            }
        }
    }
    std::set<uint32_t> ready;
    for (size_t i = 0; i < G; ++i)
        if (indeg[i] == 0) ready.insert((uint32_t)i);
    auto outside = [](const std::set<int> &a, const std::set<int> &t) {
        int k = 0;
        for (int q : a) k += t.count(q) ? 0 : 1;
        return k;
    };
    // Fill one pass starting from gate `seed` (taken first), then every
    // fitting ready gate in index order; works on copies unless `commit`.
    // Returns the gates taken.  (Seeding each pass with the ready gate whose
    // fill takes the most gates measured no better than the lowest one.)
    auto fill = [&](uint32_t seed, bool commit, std::set<int> *tile_out) -> std::vector<uint32_t> {
        std::vector<int> deg_copy;
        std::set<uint32_t> ready_copy;
        std::vector<int> &deg = commit ? indeg : (deg_copy = indeg);
        std::set<uint32_t> &rdy = commit ? ready : (ready_copy = ready);
        std::set<int> cur, sel;
        std::vector<uint32_t> taken;
        auto take = [&](uint32_t i) {
            const CGate &g = cg[gate_ids[i]];
            for (int b = 0; b < g.nq; ++b) {
                if (g.q[b] < C) continue;
                (g.mix[b] ? cur : sel).insert(g.q[b]);
            }
            taken.push_back(i);
            rdy.erase(i);
            for (uint32_t sx : succ[i])
                if (--deg[sx] == 0) rdy.insert(sx);
        };
        take(seed);
        bool grew = true;
        while (grew) {
            grew = false;
            for (uint32_t i : rdy) {
                const CGate &g = cg[gate_ids[i]];
                std::set<int> need = cur, nsel = sel;
                for (int b = 0; b < g.nq; ++b) {
                    if (g.q[b] < C) continue;
                    (g.mix[b] ? need : nsel).insert(g.q[b]);
                }
                if ((int)need.size() > jmax || outside(nsel, need) > qs::kMaxOuterSel) continue;
                take(i);
                grew = true;
                break;  // the ready set changed: rescan from the lowest index
            }
        }
        if (tile_out) *tile_out = cur;
        return taken;
    };
    std::vector<PassPlan> out;
    size_t placed = 0;
    while (placed < G) {
        const uint32_t best = *ready.begin();
        PassPlan p;
        std::set<int> cur;
        for (uint32_t i : fill(best, true, &cur)) p.gates.push_back(gate_ids[i]);
        placed += p.gates.size();
        p.tile.assign(cur.begin(), cur.end());
        out.push_back(p);
    }
    for (auto &pp : out) {
        std::set<int> s2(pp.tile.begin(), pp.tile.end());
        for (int q = pad_lo; q < pad_hi && (int)s2.size() < jmin; ++q) s2.insert(q);
        pp.tile.assign(s2.begin(), s2.end());
    }
    return out;
}

bool plan_dual_sweeps(const std::vector<CGate> &cg, const std::vector<uint32_t> &gl, const int32_t *slots,
                      const uint64_t *gen_x, const uint64_t *gen_z, const std::vector<int> &tile, int C, int RB,
                      std::vector<qs::Sweep> *all_sw, std::vector<qs::ROp> *all_rops, std::vector<cplx> *all_pool,
                      DualSweepPlan *out) {
    const int nb = C + (int)tile.size();
    if (nb < RB) return false;
    std::vector<qs::KGate> kg;
    std::vector<int32_t> sum_slot;
    std::vector<uint32_t> gid;
    int32_t ls = 0;
    for (uint32_t gi : gl) {
        const qs::KGate g = to_kgate(cg[gi], tile, C);
        if (slots[gi] >= 0) {
            kg.push_back(g);
            sum_slot.push_back(ls++);
            gid.push_back(gi);
        }
        kg.push_back(g);
        sum_slot.push_back(-1);
        gid.push_back(gi);
    }
    const auto sweeps = plan_sweeps(kg, 0, kg.size(), nb, RB);
    std::vector<RawOp> raw;
    std::vector<cplx> rpool;
    for (const auto &sw : sweeps)
        for (int i = sw.g0; i < sw.g1; ++i) {
            if (sum_slot[i] >= 0) {
                if (!build_sum_op(gen_x[gid[i]], gen_z[gid[i]], sum_slot[i], sw, RB, tile, C, &raw, &rpool))
                    return false;
            } else {
                build_gate_op(kg[i], sw, RB, &raw, &rpool);
            }
        }
    std::vector<qs::Sweep> msw;
    merge_diagonal_ops(sweeps, 0, &raw, &rpool, &msw);
    std::vector<qs::ROp> rops;
    std::vector<int> outer;
    const size_t pool0 = all_pool->size();
    if (!finalize_ops(raw, rpool, nb, &outer, &rops, all_pool)) {
        all_pool->resize(pool0);
        return false;
    }
    fuse_half_chains(&rops, 0, msw);
    out->sw_off = all_sw->size();
    out->nsw = msw.size();
    out->rop_off = all_rops->size();
    out->outer = outer;
    all_sw->insert(all_sw->end(), msw.begin(), msw.end());
    all_rops->insert(all_rops->end(), rops.begin(), rops.end());
    return true;
}

std::string format_size(unsigned long long size) {
    char buf[64];
    if (size > (1ULL << 30)) snprintf(buf, sizeof(buf), "%.3f GiB", (double)size / (1ULL << 30));
    else if (size > (1ULL << 20)) snprintf(buf, sizeof(buf), "%.3f MiB", (double)size / (1ULL << 20));
    else if (size > (1ULL << 10)) snprintf(buf, sizeof(buf), "%.3f KiB", (double)size / (1ULL << 10));
    else snprintf(buf, sizeof(buf), "%llu bytes", size);
    return buf;
}

int env_int(const char *name, int dflt) {
    const char *v = std::getenv(name);
    return v ? std::atoi(v) : dflt;
}

}  // namespace

// A failed call also leaves its error as the thread's last CUDA error; it is
// cleared here so that the next launch check does not report it again.
#define CUDA_TRY(h, expr)                                                               \
    do {                                                                                \
        cudaError_t e__ = (expr);                                                       \
        if (e__ != cudaSuccess) {                                                       \
            (void)cudaGetLastError();                                                   \
            (h)->err = std::string(#expr) + ": " + cudaGetErrorString(e__);             \
            return QS_ERR_CUDA;                                                         \
        }                                                                               \
    } while (0)

// =====================================================================
// compressed state
// =====================================================================
struct qs_state {
    uint32_t n = 0, B = 0, C = 0, nb = 0;
    uint64_t nchunks = 0;
    bool f64 = true;
    double eps_rel = 0, eps_abs = 0;
    qs::CodecParams codec{};
    uint32_t flags = 0;
    int tile_log2 = 13;
    cudaStream_t stream = nullptr;
    std::string err = "no error";

    std::vector<qs_gate> gates;
    std::vector<CGate> cgates;
    std::vector<std::vector<uint32_t>> stages;
    std::vector<std::vector<uint32_t>> b2g;
    std::vector<uint32_t> num_groups;
    bool planned = false;

    struct DevPass {
        uint32_t stage;
        int j;
        int32_t tq[qs::kMaxTileQubits];
        uint32_t gate_off, ngates;
        uint32_t sweep_off, nsweeps;
        uint32_t op_off;
        int rb;
        int nouter;
        int8_t outer_q[qs::kMaxOuterSel];
        bool first, final;
        int kind;             // 0: tile pass, 1: chunk-header permutation only
        bool code_moves;      // tile pass whose ops only move amplitudes (X / SWAP)
        qs::ChunkPerm perm;   // where the pass stores each chunk
    };
    qs::Sweep *sweeps_dev = nullptr;
    qs::ROp *ops_dev = nullptr;
    void *pool_dev = nullptr;
    std::vector<DevPass> passes;
    // Merged tail: once every block is stored, the remaining stages run as
    // one gate sequence (plan_tail_passes), planned for the first stage at
    // which that happened and kept while the circuit stays registered.
    bool merge_tail = true;
    int tail_from = -1;
    std::vector<DevPass> tail_passes;
    std::vector<int> tail_stage_end;      // per stage from tail_from: the tail pass ending it
    qs::Sweep *tail_sweeps_dev = nullptr;
    qs::ROp *tail_ops_dev = nullptr;
    void *tail_pool_dev = nullptr;
    unsigned long long *tail_stats = nullptr;  // 3 counters per tail pass
    size_t tail_stats_cap = 0;
    std::vector<cudaEvent_t> tail_ev;
    // 1 when every block is stored (mask_full_kernel): mapped pinned host
    // memory and its device alias, written by the kernel itself
    uint32_t *full_host = nullptr;
    uint32_t *full_map = nullptr;
    // end-of-apply error flag, counters, stage history and tail statistics,
    // gathered by readback_kernel into mapped pinned host memory
    unsigned long long *rb_host = nullptr;
    unsigned long long *rb_map = nullptr;
    size_t rb_cap = 0;
    int last_tail_from = -1;              // stage the last apply merged from (-1: none)
    void drop_tail() {
        if (tail_sweeps_dev) cudaFree(tail_sweeps_dev);
        if (tail_ops_dev) cudaFree(tail_ops_dev);
        if (tail_pool_dev) cudaFree(tail_pool_dev);
        for (auto e : tail_ev) cudaEventDestroy(e);
        tail_ev.clear();
        tail_sweeps_dev = nullptr;
        tail_ops_dev = nullptr;
        tail_pool_dev = nullptr;
        tail_passes.clear();
        tail_stage_end.clear();
        tail_from = -1;
    }
    std::vector<uint64_t> stage_amps;   // amplitudes in active groups (for stats), filled on demand

    qs::ChunkMeta *meta[2] = {nullptr, nullptr};
    uint32_t *arena[2] = {nullptr, nullptr};
    uint64_t capacity = 0;
    bool host_store = false;   // arenas in pinned, device-mapped host memory (QS_FLAG_HOST_STORE)
    bool staged = false;       // tile passes prefetch payloads with bulk copies (staged_pass_kernel)
    bool staged_ok = true;     // the staged kernel can run (HBM arenas): dense k-qubit passes
    unsigned long long *counters = nullptr;  // [0..1] bump, [2..4] stats, [5] init scratch, [6] header-pass bytes, [7] diagonal-pass total
    uint8_t *mask = nullptr;
    uint32_t *block_nz = nullptr;
    unsigned long long *block_bytes = nullptr, *block_acc = nullptr;
    uint8_t *group_active = nullptr;
    uint32_t *b2g_dev = nullptr;
    qs::KGate *kgates = nullptr;
    unsigned long long *history_dev = nullptr;  // [0..ns] totals, [ns+1..2ns] active blocks per stage
    size_t history_cap = 0;
    std::vector<cudaEvent_t> pass_ev;           // QS_FLAG_PROFILE: two events per pass
    int32_t *error_dev = nullptr;
    double *dscratch = nullptr;
    int cur = 0;     // payload arena in use
    int mcur = 0;    // chunk-header array in use (header-only passes flip it alone)
    uint64_t arena_used = 0;

    struct Checkpoint {
        qs::ChunkMeta *meta = nullptr;
        uint32_t *arena = nullptr;
        uint64_t arena_cap = 0, used = 0;
        uint8_t *mask = nullptr;
        unsigned long long *block_bytes = nullptr;
        std::vector<uint64_t> history;
    };
    std::vector<Checkpoint> ckpt;

    std::vector<uint64_t> history;
    double times[10] = {0};
    qs_stats st{};
    cudaEvent_t ev[2] = {nullptr, nullptr};

    ~qs_state() {
        for (int i = 0; i < 2; ++i) {
            if (meta[i]) cudaFree(meta[i]);
            if (arena[i]) {
                if (host_store) cudaFreeHost(arena[i]);
                else cudaFree(arena[i]);
            }
            if (ev[i]) cudaEventDestroy(ev[i]);
        }
        if (counters) cudaFree(counters);
        if (mask) cudaFree(mask);
        if (block_nz) cudaFree(block_nz);
        if (block_bytes) cudaFree(block_bytes);
        if (block_acc) cudaFree(block_acc);
        if (group_active) cudaFree(group_active);
        if (b2g_dev) cudaFree(b2g_dev);
        if (kgates) cudaFree(kgates);
        if (sweeps_dev) cudaFree(sweeps_dev);
        if (ops_dev) cudaFree(ops_dev);
        if (pool_dev) cudaFree(pool_dev);
        drop_tail();
        if (tail_stats) cudaFree(tail_stats);
        if (full_host) cudaFreeHost(full_host);
        if (rb_host) cudaFreeHost(rb_host);
        if (history_dev) cudaFree(history_dev);
        for (auto e : pass_ev) cudaEventDestroy(e);
        if (error_dev) cudaFree(error_dev);
        if (dscratch) cudaFree(dscratch);
        for (auto &c : ckpt) free_checkpoint(c);
    }

    static void free_checkpoint(Checkpoint &c) {
        if (c.meta) cudaFree(c.meta);
        if (c.arena) cudaFree(c.arena);
        if (c.mask) cudaFree(c.mask);
        if (c.block_bytes) cudaFree(c.block_bytes);
        c = Checkpoint();
    }

    bool quiet() const { return (flags & QS_FLAG_QUIET) != 0; }
    bool ref_controls() const { return (flags & QS_FLAG_REFERENCE_CONTROLS) != 0; }
    uint64_t chunks_per_block() const { return uint64_t(1) << (B - C); }

    // Encode |basis> into the current store: only the block holding `basis`
    // is stored, every chunk of it is zero except the one holding `basis`.
    qs_status init_basis(uint64_t basis) {
        const uint64_t blk = basis >> B;
        const uint64_t chunk = basis >> C;
        CUDA_TRY(this, cudaMemsetAsync(mask, 0, nb, stream));
        CUDA_TRY(this, cudaMemsetAsync(block_bytes, 0, nb * sizeof(unsigned long long), stream));
        CUDA_TRY(this, cudaMemsetAsync(meta[mcur] + blk * chunks_per_block(), 0,
                                       chunks_per_block() * sizeof(qs::ChunkMeta), stream));
        const int comp = (int)(2 * (basis & ((uint64_t(1) << C) - 1)));
        const int32_t q1 = f64 ? qs::quantize(1.0, codec) : qs::quantize(1.0f, codec);
        const uint32_t w = qs::bit_length((uint32_t)q1);
        std::vector<uint32_t> words(qs::payload_rows(C, w) * 32, 0u);
        const int lane = comp % 32, i = comp / 32;
        const uint64_t bitpos = (uint64_t)i * w;
        const uint64_t r = bitpos >> 5, s = bitpos & 31;
        words[r * 32 + lane] |= (uint32_t)((uint64_t)q1 << s);
        if (s + w > 32) words[(r + 1) * 32 + lane] |= (uint32_t)((uint64_t)q1 >> (32 - s));
        qs::ChunkMeta md{0, 0, w};
        CUDA_TRY(this, cudaMemcpyAsync(arena[cur], words.data(), words.size() * 4, cudaMemcpyDefault, stream));
        CUDA_TRY(this, cudaMemcpyAsync(meta[mcur] + chunk, &md, sizeof(md), cudaMemcpyHostToDevice, stream));
        const uint8_t one = 1;
        CUDA_TRY(this, cudaMemcpyAsync(mask + blk, &one, 1, cudaMemcpyHostToDevice, stream));
        const unsigned long long bytes = words.size() * 4 + chunks_per_block() * sizeof(qs::ChunkMeta);
        CUDA_TRY(this, cudaMemcpyAsync(block_bytes + blk, &bytes, sizeof(bytes), cudaMemcpyHostToDevice, stream));
        CUDA_TRY(this, cudaStreamSynchronize(stream));
        arena_used = words.size() * 4;
        history.assign(1, bytes);
        return QS_OK;
    }
};

static qs_status fail(qs_state *h, qs_status s, const std::string &msg) {
    if (h) h->err = msg;
    else g_last_error = msg;
    return s;
}

extern "C" {

const char *qs_last_error(const qs_state *h) { return h ? h->err.c_str() : g_last_error.c_str(); }

qs_status qs_codec_params(qs_dtype dtype, double eps_rel, double eps_abs, int32_t *m, int32_t *L) {
    qs::CodecParams p;
    if (!qs::codec_params(dtype == QS_COMPLEX128, eps_rel, eps_abs, &p)) {
        g_last_error = "eps_rel must lie in [2^-24, 1)";
        return QS_ERR_ARG;
    }
    if (m) *m = p.m;
    if (L) *L = p.L;
    return QS_OK;
}

qs_status qs_create(qs_state **out, uint32_t n, uint32_t block_size, qs_dtype dtype, double eps_rel,
                    double eps_abs, uint32_t flags) {
    if (!out) return fail(nullptr, QS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (dtype != QS_COMPLEX128 && dtype != QS_COMPLEX64) return fail(nullptr, QS_ERR_ARG, "unknown dtype");
    if (n > 40 || block_size > n || block_size < 4)
        return fail(nullptr, QS_ERR_ARG, "need 4 <= block_size <= n <= 40");
    qs::CodecParams cp;
    if (!qs::codec_params(dtype == QS_COMPLEX128, eps_rel, eps_abs, &cp))
        return fail(nullptr, QS_ERR_ARG, "eps_rel must lie in [2^-24, 1) (BITCOMP_REL_EB)");
    if (n - block_size > 30) return fail(nullptr, QS_ERR_ARG, "at most 2^30 blocks");
    auto *h = new (std::nothrow) qs_state();
    if (!h) return fail(nullptr, QS_ERR_NOMEM, "host allocation failed");
    h->n = n;
    h->B = block_size;
    h->C = std::min<uint32_t>(block_size, (uint32_t)env_int("QOMPSIM_CHUNK_LOG2", qs::kMaxChunkLog2));
    if (h->C < (uint32_t)qs::kMinChunkLog2 || h->C > (uint32_t)qs::kMaxChunkLog2) {
        delete h;
        return fail(nullptr, QS_ERR_ARG, "QOMPSIM_CHUNK_LOG2 must lie in [4, 8]");
    }
    h->nb = 1u << (n - block_size);
    h->nchunks = uint64_t(1) << (n - h->C);
    h->f64 = dtype == QS_COMPLEX128;
    h->eps_rel = eps_rel;
    h->eps_abs = eps_abs;
    h->codec = cp;
    if (env_int("QOMPSIM_HOST_STORE", 0)) flags |= QS_FLAG_HOST_STORE;
    h->flags = flags;
    h->host_store = (flags & QS_FLAG_HOST_STORE) != 0;
    // Tile passes run pass_kernel (three 4-warp CTAs per SM, payloads copied
    // chunk by chunk with cp.async) unless QOMPSIM_STAGED_PASS=1 selects
    // staged_pass_kernel (payloads of the next tile prefetched with bulk
    // copies), which measured 1.3-1.8x slower per pass on the QFT: its
    // registers leave one 8-warp CTA per SM, and the passes are bound by
    // the latency of their decode / sweep / quantise phases, not by memory.
    // Dense k-qubit passes always use the staged kernel (it holds the tensor
    // core operands); so that they can run, the host-store arenas (read with
    // cp.async) are excluded from it.
    h->staged = !h->host_store && env_int("QOMPSIM_STAGED_PASS", 0) != 0;
    h->staged_ok = !h->host_store;
    h->merge_tail = env_int("QOMPSIM_MERGE_TAIL", 1) != 0;
    h->tile_log2 = env_int("QOMPSIM_TILE_LOG2", h->f64 ? 12 : 13);
    h->tile_log2 = std::max<int>(h->tile_log2, (int)h->C + 2);
    h->tile_log2 = std::min<int>(h->tile_log2, std::min<int>(qs::kMaxTileLog2, (int)h->C + qs::kMaxTileQubits));

    auto cleanup = [&](qs_status s) { std::string m = h->err; delete h; g_last_error = m; return s; };
#define CREATE_TRY(expr)                                                         \
    do {                                                                         \
        cudaError_t e__ = (expr);                                                \
        if (e__ != cudaSuccess) {                                                \
            h->err = std::string(#expr) + ": " + cudaGetErrorString(e__);        \
            return cleanup(e__ == cudaErrorMemoryAllocation ? QS_ERR_CAPACITY : QS_ERR_CUDA); \
        }                                                                        \
    } while (0)

    size_t free_b = 0, total_b = 0;
    CREATE_TRY(cudaMemGetInfo(&free_b, &total_b));
    const uint64_t meta_bytes = h->nchunks * sizeof(qs::ChunkMeta);
    const uint64_t worst = h->nchunks * qs::payload_bytes((int)h->C, 32);
    const uint64_t reserve = (uint64_t)1 << 30;
    uint64_t avail = free_b > 2 * meta_bytes + reserve ? free_b - 2 * meta_bytes - reserve : 0;
    if (h->host_store) {
        // spill tier: the two payload arenas live in pinned host memory that
        // the passes read and write through the bus; headers, masks and
        // counters stay in HBM.  Default size: a quarter of the host's free
        // memory each (two arenas), at most the worst case.
        const uint64_t host_free = (uint64_t)sysconf(_SC_AVPHYS_PAGES) * (uint64_t)sysconf(_SC_PAGESIZE);
        avail = host_free / 2;
    }
    const char *cap_env = std::getenv("QOMPSIM_ARENA_BYTES");
    h->capacity = cap_env ? (uint64_t)std::strtoull(cap_env, nullptr, 10) : std::min<uint64_t>(worst, avail / 2);
    h->capacity = (h->capacity + 127) / 128 * 128;
    if (h->capacity < std::min<uint64_t>(worst, 4096)) {
        h->err = h->host_store ? "not enough host memory for the compressed store"
                               : "not enough device memory for the compressed store";
        return cleanup(QS_ERR_CAPACITY);
    }
    for (int i = 0; i < 2; ++i) {
        CREATE_TRY(cudaMalloc(&h->meta[i], meta_bytes));
        if (h->host_store) {
            void *hp = nullptr;
            CREATE_TRY(cudaHostAlloc(&hp, h->capacity, cudaHostAllocMapped | cudaHostAllocPortable));
            h->arena[i] = static_cast<uint32_t *>(hp);
            void *dp = nullptr;
            CREATE_TRY(cudaHostGetDevicePointer(&dp, hp, 0));
            if (dp != hp) {
                h->err = "mapped host arena has a different device address (no unified addressing)";
                return cleanup(QS_ERR_CUDA);
            }
        } else {
            CREATE_TRY(cudaMalloc(&h->arena[i], h->capacity));
        }
        CREATE_TRY(cudaMemset(h->meta[i], 0, meta_bytes));
        CREATE_TRY(cudaEventCreate(&h->ev[i]));
    }
    CREATE_TRY(cudaMalloc(&h->counters, 8 * sizeof(unsigned long long)));
    CREATE_TRY(cudaMalloc(&h->mask, h->nb));
    CREATE_TRY(cudaMalloc(&h->block_nz, h->nb * sizeof(uint32_t)));
    CREATE_TRY(cudaMalloc(&h->block_bytes, h->nb * sizeof(unsigned long long)));
    CREATE_TRY(cudaMalloc(&h->block_acc, h->nb * sizeof(unsigned long long)));
    CREATE_TRY(cudaMalloc(&h->group_active, h->nb));
    // 8 bytes: the end-of-apply readback copies it as one 64-bit word
    CREATE_TRY(cudaMalloc(&h->error_dev, sizeof(unsigned long long)));
    CREATE_TRY(cudaMalloc(&h->dscratch, 4 * sizeof(double)));
    CREATE_TRY(cudaMemset(h->error_dev, 0, sizeof(unsigned long long)));
#undef CREATE_TRY
    qs_status s = h->init_basis(0);
    if (s != QS_OK) return cleanup(s);
    if (!h->quiet()) {
        printf("B200 fused stage pipeline, error-bounded block codec (%s)\n", h->f64 ? "complex128" : "complex64");
        printf("  relative error bound: %g\n", eps_rel);
        printf("  absolute error bound: %g\n", eps_abs);
        fflush(stdout);
    }
    *out = h;
    return QS_OK;
}

qs_status qs_destroy(qs_state *h) {
    delete h;
    return QS_OK;
}

qs_status qs_set_stream(qs_state *h, void *stream) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    h->stream = (cudaStream_t)stream;
    return QS_OK;
}

qs_status qs_register_gates(qs_state *h, const qs_gate *gates, size_t count) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (count && !gates) return fail(h, QS_ERR_ARG, "gates is NULL");
    std::vector<CGate> cg(count);
    for (size_t i = 0; i < count; ++i) {
        std::string e;
        if (!canonicalize(gates[i], h->ref_controls(), h->n, &cg[i], &e))
            return fail(h, strnlen(gates[i].name, 24) && std::string(gates[i].name) == "FusedSWAP"
                               ? QS_ERR_UNSUPPORTED_GATE
                               : (e.find("index") != std::string::npos || e.find("duplicated") != std::string::npos
                                      ? QS_ERR_ARG
                                      : QS_ERR_UNSUPPORTED_GATE),
                        "gate " + std::to_string(i) + ": " + e);
    }
    h->gates.assign(gates, gates + count);
    h->cgates.swap(cg);
    h->planned = false;
    h->stages.clear();
    return QS_OK;
}

// partition_circuit (compressed_state.hpp:509-583).
static std::vector<std::vector<uint32_t>> partition_circuit(const qs_state *h, uint32_t inner_size) {
    std::vector<std::vector<uint32_t>> stages;
    std::vector<uint32_t> cur, global_indices, global_targets;
    const uint32_t threshold = std::max<uint32_t>(inner_size, 2u);
    for (uint32_t i = 0; i < h->gates.size(); ++i) {
        const qs_gate &g = h->gates[i];
        for (uint32_t k = 0; k < g.ntargets; ++k)
            if (g.targets[k] >= h->B) global_targets.push_back(g.targets[k]);
        for (uint32_t k = 0; k < g.ncontrols; ++k)
            if (g.controls[k] >= h->B) global_targets.push_back(g.controls[k]);
        std::vector<uint32_t> tmp = global_indices;
        for (uint32_t gt : global_targets)
            if (std::find(tmp.begin(), tmp.end(), gt) == tmp.end()) tmp.push_back(gt);
        if (tmp.size() > threshold) {
            stages.push_back(cur);
            cur.clear();
            tmp = global_targets;
            global_indices.clear();
            global_targets.clear();
        }
        global_indices = tmp;
        global_targets.clear();
        cur.push_back(i);
    }
    if (!cur.empty()) stages.push_back(cur);
    return stages;
}

// make_block_groups (compressed_state.hpp:585-671).
static void make_block_groups(qs_state *h) {
    h->b2g.assign(h->stages.size(), std::vector<uint32_t>(h->nb, 0));
    h->num_groups.assign(h->stages.size(), 1);
    for (size_t s = 0; s < h->stages.size(); ++s) {
        std::vector<bool> inner(h->n, false);
        for (uint32_t q = 0; q < h->B; ++q) inner[q] = true;
        for (uint32_t gi : h->stages[s]) {
            const qs_gate &g = h->gates[gi];
            for (uint32_t k = 0; k < g.ntargets; ++k)
                if (g.targets[k] >= h->B) inner[g.targets[k]] = true;
            for (uint32_t k = 0; k < g.ncontrols; ++k)
                if (g.controls[k] >= h->B) inner[g.controls[k]] = true;
        }
        std::vector<uint32_t> outer;
        for (uint32_t q = 0; q < h->n; ++q)
            if (!inner[q]) outer.push_back(q);
        for (uint32_t b = 0; b < h->nb; ++b) {
            uint32_t gid = 0;
            for (size_t i = 0; i < outer.size(); ++i) gid |= ((b >> (outer[i] - h->B)) & 1u) << i;
            h->b2g[s][b] = gid;
        }
        h->num_groups[s] = 1u << outer.size();
    }
}

// The device passes of every stage as host data: h->passes plus the op
// records, sweeps and matrix pool they index.  Host code only.
struct HostPlan {
    std::vector<qs::KGate> kg;
    std::vector<qs::Sweep> sw;
    std::vector<qs::ROp> ops;
    std::vector<cplx> pool;
};

// The device passes of one gate sequence (already relabelled through the
// chunk permutation P that its last pass applies), appended to *out with
// their ops, sweeps and matrices in *plan.  A sequence of chunk permutations
// only becomes one header pass.  *last_gate (when given) receives, per pass,
// the number k such that gates sg[0..k) have all been applied once the pass
// is done (passes may take commuting gates out of order).
static qs_status emit_passes(qs_state *h, uint32_t stage, const std::vector<CGate> &sg, const HostPerm &P,
                             HostPlan *plan, std::vector<qs_state::DevPass> *out, std::vector<size_t> *last_gate) {
    const int C = (int)h->C;
    const int jmax = std::min(h->tile_log2 - C, qs::kMaxTileQubits);
    // tiles are padded to the largest size: fewer tiles, each with its fixed
    // costs (headers, reservation, barriers) spread over more chunks
    const int jmin = std::min(jmax, std::max(env_int("QOMPSIM_TILE_MIN_QUBITS", jmax), qs::kRegBits - C));
    std::vector<qs::KGate> &kg = plan->kg;
    std::vector<qs::Sweep> &sw = plan->sw;
    std::vector<qs::ROp> &ops = plan->ops;
    std::vector<cplx> &pool = plan->pool;
    if (sg.empty()) {  // only chunk permutations: one header pass does the sequence
        qs_state::DevPass dp{};
        dp.stage = stage;
        dp.kind = 1;
        dp.first = dp.final = true;
        dp.perm = P.device();
        if (std::getenv("QOMPSIM_DEBUG_PLAN")) printf("stage %u: header permutation only\n", stage);
        out->push_back(dp);
        if (last_gate) last_gate->push_back(0);
        return QS_OK;
    }
    std::vector<uint32_t> ids(sg.size());
    for (size_t i = 0; i < ids.size(); ++i) ids[i] = (uint32_t)i;
    std::vector<char> placed_mark(sg.size(), 0);
    auto pl = env_int("QOMPSIM_DAG_PLAN", 1) ? plan_passes_dag(ids, sg, C, jmax, jmin, C, (int)h->B)
                                             : plan_passes(ids, sg, C, jmax, jmin, C, (int)h->B);
    for (size_t p = 0; p < pl.size(); ++p) {
        qs_state::DevPass dp{};
        dp.stage = stage;
        dp.j = (int)pl[p].tile.size();
        if (dp.j > qs::kMaxTileQubits) return fail(h, QS_ERR_ARG, "tile plan exceeds the tile size");
        for (int k = 0; k < dp.j; ++k) dp.tq[k] = pl[p].tile[k] - C;
        dp.gate_off = (uint32_t)kg.size();
        dp.ngates = (uint32_t)pl[p].gates.size();
        dp.first = p == 0;
        dp.final = p + 1 == pl.size();
        dp.kind = 0;
        dp.perm = dp.final ? P.device() : identity_perm();
        for (uint32_t gi : pl[p].gates) kg.push_back(to_kgate(sg[gi], pl[p].tile, C));
        if (last_gate) {
            // gates of sg applied once this pass is done: every gate below the
            // lowest index not yet placed (passes may take gates out of order)
            size_t upto = last_gate->empty() ? 0 : last_gate->back();
            for (uint32_t gi : pl[p].gates) placed_mark[gi] = 1;
            while (upto < sg.size() && placed_mark[upto]) ++upto;
            last_gate->push_back(upto);
        }
        const int RB = qs::kRegBits;
        dp.rb = RB;
        auto swp = plan_sweeps(kg, dp.gate_off, kg.size(), C + dp.j, RB);
        const size_t op0 = ops.size();
        std::vector<RawOp> raw;
        std::vector<cplx> rpool;
        build_ops(kg, dp.gate_off, swp, RB, &raw, &rpool);
        std::vector<qs::Sweep> merged;
        merge_diagonal_ops(swp, 0, &raw, &rpool, &merged);
        swp.swap(merged);
        std::vector<int> outer;
        if (!finalize_ops(raw, rpool, C + dp.j, &outer, &ops, &pool))
            return fail(h, QS_ERR_ARG, "a pass needs more outer selector qubits than the planner allows");
        fuse_half_chains(&ops, op0, swp);
        dp.nouter = (int)outer.size();
        for (size_t i = 0; i < outer.size(); ++i) dp.outer_q[i] = (int8_t)outer[i];
        dp.op_off = (uint32_t)op0;
        dp.sweep_off = (uint32_t)sw.size();
        // a pass of pure register moves carries codes through the tile
        dp.code_moves = env_int("QOMPSIM_CODE_MOVES", 1) != 0 && ops.size() > op0;
        for (size_t o = op0; o < ops.size() && dp.code_moves; ++o) {
            const int c = ops[o].code;
            dp.code_moves = (c >= qs::OPC_X && c < qs::OPC_X + 8) || (c >= qs::OPC_SWAP && c < qs::OPC_SWAP + 64);
        }
        if (std::getenv("QOMPSIM_DEBUG_PLAN")) {
            int kinds[5] = {0, 0, 0, 0, 0}, sel = 0, half = 0, moves = 0;
            for (size_t o = op0; o < ops.size(); ++o) {
                const int c = ops[o].code;
                const int kind = c == qs::OPC_SCALAR ? 0
                               : (c < qs::OPC_M2 || (c >= qs::OPC_ACC && c < qs::OPC_D4)) ? 1
                               : c < qs::OPC_D4 ? 2 : c < qs::OPC_M4 ? 3 : 4;
                ++kinds[kind];
                sel += ops[o].nsel;
                half += (c >= qs::OPC_D2H && c < qs::OPC_M2) || (c >= qs::OPC_ACC && c < qs::OPC_D4) ||
                        (c >= qs::OPC_D4H && c < qs::OPC_M4);
                moves += (c >= qs::OPC_X && c < qs::OPC_X + 8) || (c >= qs::OPC_SWAP && c < qs::OPC_SWAP + 64);
            }
            printf("stage %u pass %zu: j=%d gates=%u sweeps=%zu ops=%zu (scalar %d d2 %d m2 %d d4 %d m4 %d, "
                   "half-diagonal %d, moves %d, selectors %d, outer %d)%s tile=[", stage, p, dp.j, dp.ngates,
                   swp.size(), ops.size() - op0, kinds[0], kinds[1], kinds[2], kinds[3], kinds[4], half, moves,
                   sel, dp.nouter, dp.final && !P.identity() ? " +perm" : "");
            for (int t : pl[p].tile) printf(" %d", t);
            printf(" ]\n");
        }
        dp.nsweeps = (uint32_t)swp.size();
        sw.insert(sw.end(), swp.begin(), swp.end());
        out->push_back(dp);
    }
    return QS_OK;
}

static qs_status plan_device_passes(qs_state *h, HostPlan *plan) {
    const int C = (int)h->C;
    plan->kg.clear();
    plan->sw.clear();
    plan->ops.clear();
    plan->pool.clear();
    h->passes.clear();
    const bool permute = env_int("QOMPSIM_PERMUTE_CHUNKS", 1) != 0;
    for (uint32_t s = 0; s < h->stages.size(); ++s) {
        for (uint32_t gi : h->stages[s])
            if (gi >= h->cgates.size()) return fail(h, QS_ERR_ARG, "stage refers to a gate index out of range");
        std::vector<CGate> sg;
        HostPerm P((int)(h->n - h->C));
        stage_relabel(h->cgates, h->stages[s], C, permute, &sg, &P);
        qs_status st = emit_passes(h, s, sg, P, plan, &h->passes, nullptr);
        if (st != QS_OK) return st;
    }
    return QS_OK;
}

// The passes of stages [s0, end) planned as one gate sequence: once every
// block is stored, no stage boundary changes the zero mask or the active
// groups (every group is active, a stored block stays stored), so the
// stages' gates can share passes.  stage_end_pass[s - s0] is the first pass
// after which every gate of stages s0..s has been applied (-1: only chunk
// permutations so far).
static qs_status plan_tail_passes(qs_state *h, uint32_t s0, HostPlan *plan, std::vector<qs_state::DevPass> *passes,
                                  std::vector<int> *stage_end_pass) {
    const int C = (int)h->C;
    plan->kg.clear();
    plan->sw.clear();
    plan->ops.clear();
    plan->pool.clear();
    passes->clear();
    stage_end_pass->clear();
    const bool permute = env_int("QOMPSIM_PERMUTE_CHUNKS", 1) != 0;
    std::vector<uint32_t> ids;
    std::vector<size_t> stage_end;  // one past the last id of each stage in `ids`
    for (uint32_t s = s0; s < h->stages.size(); ++s) {
        ids.insert(ids.end(), h->stages[s].begin(), h->stages[s].end());
        stage_end.push_back(ids.size());
    }
    // relabel through the permutation accumulated over the whole tail, and
    // count, per stage end, the relabelled gates before it
    std::vector<CGate> sg;
    HostPerm P((int)(h->n - h->C));
    std::vector<size_t> kept_before(ids.size() + 1, 0);
    for (size_t i = 0; i < ids.size(); ++i) {
        std::vector<CGate> one;
        const std::vector<uint32_t> single(1, ids[i]);
        stage_relabel(h->cgates, single, C, permute, &one, &P);
        sg.insert(sg.end(), one.begin(), one.end());
        kept_before[i + 1] = sg.size();
    }
    std::vector<size_t> last_gate;
    qs_status st = emit_passes(h, s0, sg, P, plan, passes, &last_gate);
    if (st != QS_OK) return st;
    for (size_t k = 0; k < stage_end.size(); ++k) {
        const size_t kept = kept_before[stage_end[k]];  // relabelled gates up to this stage's end
        int pe = -1;
        for (size_t p = 0; p < passes->size(); ++p)
            if ((*passes)[p].kind == 0 && last_gate[p] >= kept) {
                pe = (int)p;
                break;
            }
        if (kept == 0) pe = -1;
        stage_end_pass->push_back(pe);
    }
    return QS_OK;
}

// Upload a host plan: op records, matrix pool, sweeps, block-to-group maps.
// Op records, matrix pool (in the state's precision) and sweeps of a host
// plan into fresh device buffers (the previous ones freed).
static qs_status upload_plan_buffers(qs_state *h, const HostPlan &plan, qs::ROp **ops_dev, void **pool_dev,
                                     qs::Sweep **sweeps_dev) {
    const std::vector<qs::Sweep> &sw = plan.sw;
    const std::vector<qs::ROp> &ops = plan.ops;
    const std::vector<cplx> &pool = plan.pool;
    if (*sweeps_dev) { cudaFree(*sweeps_dev); *sweeps_dev = nullptr; }
    if (*ops_dev) { cudaFree(*ops_dev); *ops_dev = nullptr; }
    if (*pool_dev) { cudaFree(*pool_dev); *pool_dev = nullptr; }
    if (!ops.empty()) {
        CUDA_TRY(h, cudaMalloc(ops_dev, ops.size() * sizeof(qs::ROp)));
        CUDA_TRY(h, cudaMemcpy(*ops_dev, ops.data(), ops.size() * sizeof(qs::ROp), cudaMemcpyHostToDevice));
    }
    if (!pool.empty()) {
        if (h->f64) {
            auto pv = pool_as<double>(pool);
            CUDA_TRY(h, cudaMalloc(pool_dev, pv.size() * sizeof(double)));
            CUDA_TRY(h, cudaMemcpy(*pool_dev, pv.data(), pv.size() * sizeof(double), cudaMemcpyHostToDevice));
        } else {
            auto pv = pool_as<float>(pool);
            CUDA_TRY(h, cudaMalloc(pool_dev, pv.size() * sizeof(float)));
            CUDA_TRY(h, cudaMemcpy(*pool_dev, pv.data(), pv.size() * sizeof(float), cudaMemcpyHostToDevice));
        }
    }
    if (!sw.empty()) {
        CUDA_TRY(h, cudaMalloc(sweeps_dev, sw.size() * sizeof(qs::Sweep)));
        CUDA_TRY(h, cudaMemcpy(*sweeps_dev, sw.data(), sw.size() * sizeof(qs::Sweep), cudaMemcpyHostToDevice));
    }
    return QS_OK;
}

static qs_status upload_device_plan(qs_state *h, const HostPlan &plan) {
    const std::vector<qs::Sweep> &sw = plan.sw;
    const std::vector<qs::ROp> &ops = plan.ops;
    if (h->kgates) { cudaFree(h->kgates); h->kgates = nullptr; }
    qs_status us = upload_plan_buffers(h, plan, &h->ops_dev, &h->pool_dev, &h->sweeps_dev);
    if (us != QS_OK) return us;
    h->drop_tail();
    if (h->b2g_dev) { cudaFree(h->b2g_dev); h->b2g_dev = nullptr; }
    if (h->history_dev) { cudaFree(h->history_dev); h->history_dev = nullptr; }
    const size_t ns = h->stages.size();
    if (ns) {
        CUDA_TRY(h, cudaMalloc(&h->b2g_dev, ns * h->nb * sizeof(uint32_t)));
        for (size_t s = 0; s < ns; ++s)
            CUDA_TRY(h, cudaMemcpy(h->b2g_dev + s * h->nb, h->b2g[s].data(), h->nb * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice));
        uint32_t gmax = *std::max_element(h->num_groups.begin(), h->num_groups.end());
        if (gmax > h->nb) return fail(h, QS_ERR_ARG, "num_groups larger than the number of blocks");
    }
    h->st.sweeps = sw.size();
    h->st.ops = ops.size();
    h->history_cap = 2 * ns + 1;
    CUDA_TRY(h, cudaMalloc(&h->history_dev, h->history_cap * sizeof(unsigned long long)));
    for (auto e : h->pass_ev) cudaEventDestroy(e);
    h->pass_ev.clear();
    if (h->flags & QS_FLAG_PROFILE) {
        h->pass_ev.resize(2 * h->passes.size());
        for (auto &e : h->pass_ev) CUDA_TRY(h, cudaEventCreate(&e));
    }
    h->planned = true;
    return QS_OK;
}

// Device-side plan: passes of every stage, gates with tile positions, maps.
static qs_status build_device_plan(qs_state *h) {
    HostPlan plan;
    qs_status st = plan_device_passes(h, &plan);
    if (st != QS_OK) return st;
    return upload_device_plan(h, plan);
}

qs_status qs_partition(qs_state *h, uint32_t inner_size, int verbose) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    for (const auto &g : h->gates)
        if (std::string(g.name, strnlen(g.name, 24)) == "FusedSWAP")
            return fail(h, QS_ERR_UNSUPPORTED_GATE, "FusedSWAP needs MPI ranks");
    h->stages = partition_circuit(h, inner_size);
    make_block_groups(h);
    qs_status s = build_device_plan(h);
    if (s != QS_OK) return s;
    if (verbose > 0) {
        printf("Circuit Stages: [");
        for (size_t i = 0; i < h->stages.size(); ++i)
            printf("%zu%s", h->stages[i].size(), i + 1 == h->stages.size() ? "" : ", ");
        printf("]\n");
    }
    if (verbose > 1) {
        printf("\n=== Block Groups ===\n");
        for (size_t s2 = 0; s2 < h->stages.size(); ++s2) {
            printf("Stage %zu block groups:\n", s2);
            std::vector<std::vector<uint32_t>> groups(h->num_groups[s2]);
            for (uint32_t b = 0; b < h->nb; ++b) groups[h->b2g[s2][b]].push_back(b);
            for (size_t g = 0; g < groups.size(); ++g) {
                printf("  Group %zu: [", g);
                for (size_t i = 0; i < groups[g].size(); ++i)
                    printf("%u%s", groups[g][i], i + 1 == groups[g].size() ? "" : ", ");
                printf("]\n");
            }
        }
    }
    fflush(stdout);
    return QS_OK;
}

qs_status qs_register_stages(qs_state *h, const uint32_t *stage_sizes, size_t nstages, const uint32_t *ids,
                             const uint32_t *block_to_group, const uint32_t *num_groups) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (nstages && (!stage_sizes || !block_to_group || !num_groups)) return fail(h, QS_ERR_ARG, "NULL argument");
    h->stages.assign(nstages, {});
    size_t off = 0;
    for (size_t s = 0; s < nstages; ++s) {
        if (stage_sizes[s] && !ids) return fail(h, QS_ERR_ARG, "stage_gate_ids is NULL");
        h->stages[s].assign(ids + off, ids + off + stage_sizes[s]);
        off += stage_sizes[s];
    }
    h->b2g.assign(nstages, std::vector<uint32_t>(h->nb));
    h->num_groups.assign(num_groups, num_groups + nstages);
    for (size_t s = 0; s < nstages; ++s) {
        for (uint32_t b = 0; b < h->nb; ++b) {
            const uint32_t g = block_to_group[s * h->nb + b];
            if (g >= h->num_groups[s]) return fail(h, QS_ERR_ARG, "group id out of range");
            h->b2g[s][b] = g;
        }
    }
    return build_device_plan(h);
}

qs_status qs_plan_stages(const qs_gate *gates, size_t count, uint32_t n, uint32_t block_size, uint32_t inner_size,
                         size_t *nstages, uint32_t *stage_sizes, uint32_t *stage_gate_ids, uint32_t *block_to_group,
                         uint32_t *num_groups) {
    if (!nstages || (count && !gates)) return fail(nullptr, QS_ERR_ARG, "NULL argument");
    if (n > 40 || block_size > n || n - block_size > 30) return fail(nullptr, QS_ERR_ARG, "bad geometry");
    qs_state tmp;  // host-only: no device allocation happens for a default state
    tmp.n = n;
    tmp.B = block_size;
    tmp.nb = 1u << (n - block_size);
    tmp.gates.assign(gates, gates + count);
    for (size_t i = 0; i < count; ++i) {
        for (uint32_t k = 0; k < gates[i].ntargets && k < 2; ++k)
            if (gates[i].targets[k] >= n) return fail(nullptr, QS_ERR_ARG, "gate target index out of range");
        for (uint32_t k = 0; k < gates[i].ncontrols && k < 2; ++k)
            if (gates[i].controls[k] >= n) return fail(nullptr, QS_ERR_ARG, "gate control index out of range");
    }
    tmp.stages = partition_circuit(&tmp, inner_size);
    make_block_groups(&tmp);
    *nstages = tmp.stages.size();
    size_t off = 0;
    for (size_t s = 0; s < tmp.stages.size(); ++s) {
        if (stage_sizes) stage_sizes[s] = (uint32_t)tmp.stages[s].size();
        if (stage_gate_ids)
            for (uint32_t g : tmp.stages[s]) stage_gate_ids[off++] = g;
        if (block_to_group) std::memcpy(block_to_group + s * tmp.nb, tmp.b2g[s].data(), tmp.nb * sizeof(uint32_t));
        if (num_groups) num_groups[s] = tmp.num_groups[s];
    }
    return QS_OK;
}

qs_status qs_stage_chunk_permutation(const qs_gate *gates, size_t count, uint32_t n, uint32_t chunk_log2,
                                     int reference_controls, qs_gate *out, size_t *out_count, int32_t *perm_dst,
                                     uint64_t *perm_flip) {
    if ((count && !gates) || !out_count || !perm_flip) return fail(nullptr, QS_ERR_ARG, "NULL argument");
    if (n > 40 || chunk_log2 > n) return fail(nullptr, QS_ERR_ARG, "bad geometry");
    std::vector<CGate> cg(count);
    std::vector<uint32_t> ids(count);
    for (size_t i = 0; i < count; ++i) {
        std::string err;
        if (!canonicalize(gates[i], reference_controls != 0, n, &cg[i], &err)) return fail(nullptr, QS_ERR_ARG, err);
        ids[i] = (uint32_t)i;
    }
    std::vector<CGate> sg;
    HostPerm P((int)(n - chunk_log2));
    stage_relabel(cg, ids, (int)chunk_log2, true, &sg, &P);
    *out_count = sg.size();
    if (out) {
        for (size_t i = 0; i < sg.size(); ++i) {
            qs_gate g;
            std::memset(&g, 0, sizeof(g));
            std::snprintf(g.name, sizeof(g.name), "DenseMatrix");
            g.ntargets = (uint32_t)sg[i].nq;
            const int dim = 1 << sg[i].nq;
            for (int k = 0; k < sg[i].nq; ++k) g.targets[k] = (uint32_t)sg[i].q[k];
            for (int k = 0; k < dim * dim; ++k) {
                g.matrix[2 * k] = sg[i].m[k].real();
                g.matrix[2 * k + 1] = sg[i].m[k].imag();
            }
            out[i] = g;
        }
    }
    if (perm_dst)
        for (size_t b = 0; b < P.dst.size(); ++b) perm_dst[b] = P.dst[b];
    *perm_flip = P.x;
    return QS_OK;
}

qs_status qs_get_plan_info(qs_state *h, uint32_t *nstages, uint32_t *nblocks) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (nstages) *nstages = (uint32_t)h->stages.size();
    if (nblocks) *nblocks = h->nb;
    return QS_OK;
}

qs_status qs_get_stage(qs_state *h, uint32_t stage, uint32_t *gate_ids, uint32_t cap, uint32_t *count,
                       uint32_t *block_to_group, uint32_t *num_groups) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (stage >= h->stages.size()) return fail(h, QS_ERR_ARG, "stage out of range");
    const auto &st = h->stages[stage];
    if (count) *count = (uint32_t)st.size();
    if (gate_ids)
        for (uint32_t i = 0; i < std::min<uint32_t>(cap, (uint32_t)st.size()); ++i) gate_ids[i] = st[i];
    if (block_to_group) std::memcpy(block_to_group, h->b2g[stage].data(), h->nb * sizeof(uint32_t));
    if (num_groups) *num_groups = h->num_groups[stage];
    return QS_OK;
}

qs_status qs_apply_circuit(qs_state *h) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (!h->planned) return fail(h, QS_ERR_STATE, "no registered circuit: call qs_partition or qs_register_stages");
    cudaStream_t s = h->stream;
    const int C = (int)h->C;
    const size_t ns = h->stages.size();
    if (!h->quiet()) {
        printf("# of PUs per rank: 1\n# of streams per PU: 1\n");
        fflush(stdout);
    }
    if (h->merge_tail && !h->full_host) {
        void *dp = nullptr;
        CUDA_TRY(h, cudaHostAlloc(&h->full_host, sizeof(uint32_t), cudaHostAllocMapped));
        CUDA_TRY(h, cudaHostGetDevicePointer(&dp, h->full_host, 0));
        h->full_map = static_cast<uint32_t *>(dp);
    }
    CUDA_TRY(h, cudaMemsetAsync(h->counters, 0, 8 * sizeof(unsigned long long), s));
    CUDA_TRY(h, cudaMemsetAsync(h->history_dev, 0, h->history_cap * sizeof(unsigned long long), s));
    CUDA_TRY(h, cudaMemsetAsync(h->error_dev, 0, sizeof(int32_t), s));
    CUDA_TRY(h, qs::launch_sum_mask_bytes(h->mask, h->block_bytes, h->nb, h->history_dev, s));
    CUDA_TRY(h, cudaEventRecord(h->ev[0], s));
    bool tile_passes = false;
    uint64_t executed = 0, executed_perm = 0, executed_codes = 0;

    // one device pass of stage map b2g (tile pass or chunk-header pass)
    auto launch_one = [&](const qs_state::DevPass &dp, const uint32_t *b2g, const qs::ROp *ops_dev,
                          const void *pool_dev, const qs::Sweep *sweeps_dev, unsigned long long *stats,
                          cudaEvent_t e0, cudaEvent_t e1) -> qs_status {
        ++executed;
        if (dp.kind == 1) {
            ++executed_perm;
            qs::PermPassArgs pa{};
            pa.B = (int)h->B;
            pa.C = C;
            pa.nchunks = h->nchunks;
            pa.meta_in = h->meta[h->mcur];
            pa.meta_out = h->meta[h->mcur ^ 1];
            pa.block_to_group = b2g;
            pa.group_active = h->group_active;
            pa.mask = h->mask;
            pa.first_pass = dp.first;
            pa.final_pass = dp.final;
            pa.block_nz = h->block_nz;
            pa.block_bytes = h->block_acc;
            pa.stats = h->counters + 6;
            pa.perm = dp.perm;
            if (e0) CUDA_TRY(h, cudaEventRecord(e0, s));
            CUDA_TRY(h, qs::launch_perm_pass(pa, s));
            if (e1) CUDA_TRY(h, cudaEventRecord(e1, s));
            h->mcur ^= 1;
            return QS_OK;
        }
        executed_codes += dp.code_moves ? 1 : 0;
        const int out = h->cur ^ 1;
        tile_passes = true;
        CUDA_TRY(h, cudaMemsetAsync(h->counters + out, 0, sizeof(unsigned long long), s));
        qs::PassArgs a{};
        a.n = (int)h->n;
        a.B = (int)h->B;
        a.C = C;
        a.j = dp.j;
        for (int k = 0; k < dp.j; ++k) a.tq[k] = dp.tq[k];
        a.n_tiles = uint64_t(1) << (h->n - C - dp.j);
        a.ops = ops_dev + dp.op_off;
        a.pool = pool_dev;
        a.sweeps = sweeps_dev + dp.sweep_off;
        a.nsweeps = (int)dp.nsweeps;
        a.rb = dp.rb;
        a.nouter = dp.nouter;
        for (int k = 0; k < qs::kMaxOuterSel; ++k) a.outer_q[k] = dp.outer_q[k];
        a.codec = h->codec;
        a.meta_in = h->meta[h->mcur];
        a.arena_in = h->arena[h->cur];
        a.meta_out = h->meta[h->mcur ^ 1];
        a.arena_out = h->arena[out];
        a.perm = dp.perm;
        a.bump = h->counters + out;
        a.capacity = h->capacity;
        a.block_to_group = b2g;
        a.group_active = h->group_active;
        a.mask = h->mask;
        a.first_pass = dp.first;
        a.final_pass = dp.final;
        a.exact_zero = (h->flags & QS_FLAG_EXACT_ZERO_TEST) ? 1 : 0;
        a.code_moves = dp.code_moves ? 1 : 0;
        // complex64: passes of several sweeps measured faster with eight
        // headers per batch, single-sweep (codec-bound) passes with four
        a.header_batch = (!h->f64 && dp.nsweeps >= 2) ? 8 : 4;
        a.block_nz = h->block_nz;
        a.block_bytes = h->block_acc;
        a.error = h->error_dev;
        a.stats = stats;
        a.staged = h->staged ? 1 : 0;
        if (e0) CUDA_TRY(h, cudaEventRecord(e0, s));
        CUDA_TRY(h, qs::launch_pass(h->f64, a, h->tile_log2, s));
        if (e1) CUDA_TRY(h, cudaEventRecord(e1, s));
        h->cur = out;
        h->mcur ^= 1;
        return QS_OK;
    };

    // whether every block is stored now (one synchronisation)
    auto mask_full_now = [&](bool *full) -> qs_status {
        // the previous flag test ended with a synchronisation, so no kernel
        // writes the flag while the host sets it
        *reinterpret_cast<volatile uint32_t *>(h->full_host) = 1u;
        CUDA_TRY(h, qs::launch_mask_full(h->mask, h->nb, h->full_map, s));
        CUDA_TRY(h, cudaStreamSynchronize(s));
        *full = *reinterpret_cast<volatile uint32_t *>(h->full_host) != 0;
        return QS_OK;
    };

    int merged_from = -1;
    size_t pi = 0;
    for (uint32_t st = 0; st < ns; ++st) {
        // every block stored: the remaining stages (two or more) share passes
        if (h->merge_tail && ns - st >= 2) {
            bool full = false;
            qs_status q = mask_full_now(&full);
            if (q != QS_OK) return q;
            if (full) {
                merged_from = (int)st;
                break;
            }
        }
        const uint32_t *b2g = h->b2g_dev + (size_t)st * h->nb;
        CUDA_TRY(h, qs::launch_stage_begin(b2g, h->mask, h->nb, h->group_active, h->num_groups[st], h->block_nz,
                                           h->block_acc, h->history_dev + ns + 1 + st, s));
        for (; pi < h->passes.size() && h->passes[pi].stage == st; ++pi) {
            const bool prof = !h->pass_ev.empty();
            qs_status q = launch_one(h->passes[pi], b2g, h->ops_dev, h->pool_dev, h->sweeps_dev, h->counters + 2,
                                     prof ? h->pass_ev[2 * pi] : nullptr, prof ? h->pass_ev[2 * pi + 1] : nullptr);
            if (q != QS_OK) return q;
        }
        CUDA_TRY(h, qs::launch_stage_end(b2g, h->group_active, h->nb, h->block_nz, h->block_acc, h->mask,
                                         h->block_bytes, h->history_dev + st + 1, s));
    }
    const size_t main_passes = pi;
    size_t ntail = 0;
    if (merged_from >= 0) {
        if (h->tail_from != merged_from) {
            HostPlan plan;
            std::vector<qs_state::DevPass> tp;
            std::vector<int> tend;
            qs_status q = plan_tail_passes(h, (uint32_t)merged_from, &plan, &tp, &tend);
            if (q != QS_OK) return q;
            q = upload_plan_buffers(h, plan, &h->tail_ops_dev, &h->tail_pool_dev, &h->tail_sweeps_dev);
            if (q != QS_OK) return q;
            for (auto e : h->tail_ev) cudaEventDestroy(e);
            h->tail_ev.clear();
            if (h->flags & QS_FLAG_PROFILE) {
                h->tail_ev.resize(2 * tp.size());
                for (auto &e : h->tail_ev) CUDA_TRY(h, cudaEventCreate(&e));
            }
            if (h->tail_stats_cap < 3 * tp.size()) {
                if (h->tail_stats) cudaFree(h->tail_stats);
                h->tail_stats = nullptr;
                h->tail_stats_cap = 0;
                CUDA_TRY(h, cudaMalloc(&h->tail_stats, 3 * tp.size() * sizeof(unsigned long long)));
                h->tail_stats_cap = 3 * tp.size();
            }
            h->tail_passes.swap(tp);
            h->tail_stage_end.swap(tend);
            h->tail_from = merged_from;
        }
        ntail = h->tail_passes.size();
        // the last stage's map and group flags serve the whole tail (every
        // group is active); its begin/end bracket the tail's passes
        const uint32_t last = (uint32_t)ns - 1;
        const uint32_t *b2g = h->b2g_dev + (size_t)last * h->nb;
        CUDA_TRY(h, qs::launch_stage_begin(b2g, h->mask, h->nb, h->group_active, h->num_groups[last], h->block_nz,
                                           h->block_acc, h->history_dev + ns + 1 + last, s));
        CUDA_TRY(h, cudaMemsetAsync(h->tail_stats, 0, 3 * ntail * sizeof(unsigned long long), s));
        for (size_t p = 0; p < ntail; ++p) {
            const bool prof = !h->tail_ev.empty();
            qs_status q = launch_one(h->tail_passes[p], b2g, h->tail_ops_dev, h->tail_pool_dev, h->tail_sweeps_dev,
                                     h->tail_stats + 3 * p, prof ? h->tail_ev[2 * p] : nullptr,
                                     prof ? h->tail_ev[2 * p + 1] : nullptr);
            if (q != QS_OK) return q;
        }
        CUDA_TRY(h, qs::launch_stage_end(b2g, h->group_active, h->nb, h->block_nz, h->block_acc, h->mask,
                                         h->block_bytes, h->history_dev + last + 1, s));
    }
    CUDA_TRY(h, cudaEventRecord(h->ev[1], s));
    // error flag, counters, stage history and tail statistics reach the host
    // through mapped memory written by one kernel: no copy-engine transfer
    // that would queue behind another stream's store export
    const size_t rb_words = 1 + 8 + h->history_cap + 3 * ntail;
    if (h->rb_cap < rb_words) {
        CUDA_TRY(h, cudaStreamSynchronize(s));
        if (h->rb_host) cudaFreeHost(h->rb_host);
        h->rb_host = h->rb_map = nullptr;
        h->rb_cap = 0;
        void *dp = nullptr;
        CUDA_TRY(h, cudaHostAlloc(&h->rb_host, rb_words * sizeof(unsigned long long), cudaHostAllocMapped));
        CUDA_TRY(h, cudaHostGetDevicePointer(&dp, h->rb_host, 0));
        h->rb_map = static_cast<unsigned long long *>(dp);
        h->rb_cap = rb_words;
    }
    qs::ReadbackList rl{};
    rl.src[0] = reinterpret_cast<const unsigned long long *>(h->error_dev);
    rl.words[0] = 1;
    rl.src[1] = h->counters;
    rl.words[1] = 8;
    rl.src[2] = h->history_dev;
    rl.words[2] = h->history_cap;
    rl.n = 3;
    if (ntail) {
        rl.src[3] = h->tail_stats;
        rl.words[3] = 3 * ntail;
        rl.n = 4;
    }
    CUDA_TRY(h, qs::launch_readback(rl, h->rb_map, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    const volatile unsigned long long *rb = h->rb_host;
    const int32_t errflag = (int32_t)(uint32_t)(rb[0] & 0xffffffffull);
    unsigned long long ctr[8];
    for (int i = 0; i < 8; ++i) ctr[i] = rb[1 + i];
    std::vector<unsigned long long> hist(h->history_cap);
    for (size_t i = 0; i < hist.size(); ++i) hist[i] = rb[9 + i];
    std::vector<unsigned long long> tstats(3 * ntail);
    for (size_t i = 0; i < tstats.size(); ++i) tstats[i] = rb[9 + h->history_cap + i];
    float ms = 0;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    if (errflag == 2)
        return fail(h, QS_ERR_TIMEOUT,
                    "a pass gave up waiting for its staged chunk payloads (bounded wait); the state is invalid");
    if (errflag)
        return fail(h, QS_ERR_CAPACITY,
                    "compressed store overflowed its arena (" + std::to_string(h->capacity) +
                        " bytes); the state is invalid.  Set QOMPSIM_ARENA_BYTES larger.");
    if (tile_passes) h->arena_used = ctr[h->cur];
    // stages inside the merged tail: every block active; the stored total at
    // a stage's end is the store written by the tail pass that applied the
    // stage's last gate (every tail pass rewrites the whole store)
    if (merged_from >= 0) {
        for (size_t st = (size_t)merged_from; st + 1 < ns; ++st) {
            hist[ns + 1 + st] = h->nb;
            const int pe = h->tail_stage_end[st - (size_t)merged_from];
            hist[st + 1] = pe >= 0 ? tstats[3 * (size_t)pe + 1] : hist[st];
        }
    }
    h->history.assign(hist.begin(), hist.begin() + ns + 1);
    uint64_t updates = 0;
    for (size_t st = 0; st < ns; ++st) updates += (uint64_t)h->stages[st].size() * hist[ns + 1 + st] << h->B;
    double pass_ms = 0, perm_ms = 0;
    const bool print_passes = std::getenv("QOMPSIM_DEBUG_PASS_MS") != nullptr;
    auto account = [&](const qs_state::DevPass &dp, cudaEvent_t e0, cudaEvent_t e1, const char *tag,
                       size_t p) -> qs_status {
        float t = 0;
        CUDA_TRY(h, cudaEventElapsedTime(&t, e0, e1));
        (dp.kind == 1 ? perm_ms : pass_ms) += t;
        if (print_passes)
            printf("%spass %zu stage %u kind %d j %d gates %u sweeps %u codes %d ms %.3f\n", tag, p, dp.stage, dp.kind,
                   dp.j, dp.ngates, dp.nsweeps, dp.code_moves ? 1 : 0, t);
        return QS_OK;
    };
    if (!h->pass_ev.empty())
        for (size_t p = 0; p < main_passes; ++p) {
            qs_status q = account(h->passes[p], h->pass_ev[2 * p], h->pass_ev[2 * p + 1], "", p);
            if (q != QS_OK) return q;
        }
    if (!h->tail_ev.empty())
        for (size_t p = 0; p < ntail; ++p) {
            qs_status q = account(h->tail_passes[p], h->tail_ev[2 * p], h->tail_ev[2 * p + 1], "tail ", p);
            if (q != QS_OK) return q;
        }
    if (print_passes) fflush(stdout);
    unsigned long long rd = ctr[2], wr = ctr[3], tiles = ctr[4];
    for (size_t p = 0; p < ntail; ++p) {
        rd += tstats[3 * p];
        wr += tstats[3 * p + 1];
        tiles += tstats[3 * p + 2];
    }
    h->times[1] += ms / 1000.0;
    h->st.stages = ns;
    h->st.passes = executed;
    h->st.bytes_read = rd;
    h->st.bytes_written = wr;
    h->st.tiles = tiles;
    h->st.amp_gate_updates = updates;
    h->st.kernel_ms = (h->pass_ev.empty() && h->tail_ev.empty()) ? ms : pass_ms;
    h->st.apply_ms = ms;
    h->st.mantissa_bits = h->codec.m;
    h->st.linear_exp = h->codec.L;
    h->st.chunk_log2 = (int32_t)h->C;
    h->st.tile_log2 = h->tile_log2;
    h->st.perm_passes = executed_perm;
    h->st.code_move_passes = executed_codes;
    h->st.perm_bytes = ctr[6];
    h->st.perm_ms = perm_ms;
    h->st.merged_from = merged_from;
    h->st.tail_passes = ntail;
    h->last_tail_from = merged_from;
    if (!h->quiet()) {
        printf("Total SV bytes: %s\n", format_size(hist[0]).c_str());
        for (size_t st = 0; st < ns; ++st)
            printf("[Stage %zu/%zu] Total SV bytes: %s\n", st, ns - 1, format_size(hist[st + 1]).c_str());
        fflush(stdout);
    }
    return QS_OK;
}

qs_status qs_norm_squared(qs_state *h, double *out) {
    if (!h || !out) return fail(h, QS_ERR_ARG, "NULL argument");
    CUDA_TRY(h, cudaMemsetAsync(h->dscratch, 0, sizeof(double), h->stream));
    CUDA_TRY(h, qs::launch_norm(h->f64, h->meta[h->mcur], h->arena[h->cur], h->mask, (int)h->B, (int)h->C, h->codec,
                                h->nchunks, h->dscratch, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(out, h->dscratch, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_get_vector(qs_state *h, double *out, int renormalize) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    return qs_get_amplitudes(h, 0, uint64_t(1) << h->n, out, renormalize);
}

qs_status qs_get_amplitudes(qs_state *h, uint64_t first, uint64_t count, double *out, int renormalize) {
    if (!h || (count && !out)) return fail(h, QS_ERR_ARG, "NULL argument");
    const uint64_t chunk_amps = uint64_t(1) << h->C;
    const uint64_t dim = uint64_t(1) << h->n;
    if (first > dim || count > dim - first) return fail(h, QS_ERR_ARG, "amplitude range outside the state");
    if ((first | count) & (chunk_amps - 1))
        return fail(h, QS_ERR_ARG, "first and count must be multiples of 2^chunk_log2 (qs_get_stats)");
    double scale = 1.0;
    if (renormalize) {
        double nrm = 0;
        qs_status s = qs_norm_squared(h, &nrm);
        if (s != QS_OK) return s;
        if (nrm > 0) scale = 1.0 / std::sqrt(nrm);
    }
    const uint64_t cfirst = first / chunk_amps, ccount = count / chunk_amps;
    if (!ccount) return QS_OK;
    const uint64_t slab_chunks = std::max<uint64_t>(1, (uint64_t(1) << 24) / chunk_amps);
    double *dbuf = nullptr;
    const uint64_t nslab = std::min<uint64_t>(slab_chunks, ccount);
    CUDA_TRY(h, cudaMalloc(&dbuf, nslab * chunk_amps * 2 * sizeof(double)));
    qs_status rs = QS_OK;
    for (uint64_t c0 = 0; c0 < ccount; c0 += nslab) {
        const uint64_t cnt = std::min<uint64_t>(nslab, ccount - c0);
        cudaError_t e = qs::launch_readout(h->f64, h->meta[h->mcur], h->arena[h->cur], h->mask, (int)h->B, (int)h->C,
                                           h->codec, cfirst + c0, cnt, dbuf, scale, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out + c0 * chunk_amps * 2, dbuf, cnt * chunk_amps * 2 * sizeof(double),
                                cudaMemcpyDefault, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            h->err = std::string("readout: ") + cudaGetErrorString(e);
            rs = QS_ERR_CUDA;
            break;
        }
    }
    cudaFree(dbuf);
    return rs;
}

// Block-wise sampling of CompressedQuantumState::sampling_blockwise
// (compressed_state.hpp:1600-1681) for one rank: the sequential FP64 block
// masses and the within-block inverse-cdf searches run on the device
// (launch_block_mass / launch_sample_in_block); the shot split, the uniform
// draws and the final shuffle use the reference's generators
// (std::mt19937_64 seeded with seed and with seed + 1, the binomial and
// uniform distributions, std::shuffle) in its order, so the same decoded
// amplitudes give the same samples.
qs_status qs_sample_blockwise(qs_state *h, uint32_t n_shots, uint32_t seed, uint64_t *out) {
    if (!h || (n_shots && !out)) return fail(h, QS_ERR_ARG, "NULL argument");
    struct DevTmp {
        void *p[5] = {};
        ~DevTmp() {
            for (void *q : p)
                if (q) cudaFree(q);
        }
    } tmp;
    double *prefix = nullptr, *bmass = nullptr, *rin = nullptr;
    uint32_t *sblock = nullptr;
    uint64_t *dout = nullptr;
    CUDA_TRY(h, cudaMalloc(&prefix, h->nchunks * sizeof(double)));
    tmp.p[0] = prefix;
    CUDA_TRY(h, cudaMalloc(&bmass, h->nb * sizeof(double)));
    tmp.p[1] = bmass;
    CUDA_TRY(h, qs::launch_block_mass(h->f64, h->meta[h->mcur], h->arena[h->cur], h->mask, (int)h->B, (int)h->C,
                                      h->codec, h->nb, prefix, bmass, h->stream));
    std::vector<double> mass(h->nb);
    CUDA_TRY(h, cudaMemcpyAsync(mass.data(), bmass, h->nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    double total = 0.0;
    for (double m : mass) total += m;
    if (!(total > 0.0) || !std::isfinite(total))
        return fail(h, QS_ERR_DOMAIN,
                    "CompressedQuantumState::sampling_blockwise: state has no finite positive probability mass");
    std::mt19937_64 rng(seed);
    std::vector<uint32_t> shots(mass.size(), 0);
    uint32_t left = n_shots;
    double rest = total;
    for (size_t g = 0; g < mass.size() && left > 0; g++) {
        const double pg = rest > 0 ? std::min(1.0, mass[g] / rest) : 0.0;
        std::binomial_distribution<uint32_t> bin(left, pg);
        const uint32_t k = (g + 1 == mass.size()) ? left : bin(rng);
        shots[g] = k;
        left -= k;
        rest -= mass[g];
    }
    // rank 0 of the reference: its local generator is seeded with seed + 1
    // in 32-bit arithmetic
    std::mt19937_64 rng_local(static_cast<uint32_t>(seed + 1u));
    std::uniform_real_distribution<double> uni(0.0, 1.0);
    std::vector<uint32_t> hb;
    std::vector<double> hr;
    hb.reserve(n_shots);
    hr.reserve(n_shots);
    for (uint32_t b = 0; b < h->nb; b++)
        for (uint32_t s = 0; s < shots[b]; s++) {
            hb.push_back(b);
            hr.push_back(uni(rng_local) * mass[b]);
        }
    const uint64_t ns = hb.size();
    std::vector<uint64_t> mine(ns);
    if (ns) {
        CUDA_TRY(h, cudaMalloc(&sblock, ns * sizeof(uint32_t)));
        tmp.p[2] = sblock;
        CUDA_TRY(h, cudaMalloc(&rin, ns * sizeof(double)));
        tmp.p[3] = rin;
        CUDA_TRY(h, cudaMalloc(&dout, ns * sizeof(uint64_t)));
        tmp.p[4] = dout;
        CUDA_TRY(h, cudaMemcpyAsync(sblock, hb.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(rin, hr.data(), ns * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(h, qs::launch_sample_in_block(h->f64, h->meta[h->mcur], h->arena[h->cur], h->mask, (int)h->B,
                                               (int)h->C, h->codec, prefix, bmass, sblock, rin, ns, dout,
                                               h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(mine.data(), dout, ns * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    std::shuffle(mine.begin(), mine.end(), rng);
    if (ns) std::memcpy(out, mine.data(), ns * sizeof(uint64_t));
    return QS_OK;
}

qs_status qs_get_zero_mask(qs_state *h, uint8_t *out) {
    if (!h || !out) return fail(h, QS_ERR_ARG, "NULL argument");
    CUDA_TRY(h, cudaMemcpyAsync(out, h->mask, h->nb, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_get_block_bytes(qs_state *h, uint64_t *out) {
    if (!h || !out) return fail(h, QS_ERR_ARG, "NULL argument");
    CUDA_TRY(h, cudaMemcpyAsync(out, h->block_bytes, h->nb * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_get_max_sv_bytes(qs_state *h, uint64_t *out) {
    if (!h || !out) return fail(h, QS_ERR_ARG, "NULL argument");
    uint64_t m = 0;
    for (uint64_t v : h->history) m = std::max(m, v);
    *out = m;
    return QS_OK;
}

qs_status qs_get_sv_bytes_history(qs_state *h, uint64_t *out, size_t cap, size_t *count) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (count) *count = h->history.size();
    if (out)
        for (size_t i = 0; i < std::min(cap, h->history.size()); ++i) out[i] = h->history[i];
    return QS_OK;
}

qs_status qs_get_total_times(qs_state *h, double out[10]) {
    if (!h || !out) return fail(h, QS_ERR_ARG, "NULL argument");
    for (int i = 0; i < 10; ++i) out[i] = h->times[i];
    (void)kTimerKeys;
    return QS_OK;
}

qs_status qs_get_stats(qs_state *h, qs_stats *out) {
    if (!h || !out) return fail(h, QS_ERR_ARG, "NULL argument");
    *out = h->st;
    // the state's geometry and codec hold before any apply
    out->mantissa_bits = h->codec.m;
    out->linear_exp = h->codec.L;
    out->chunk_log2 = (int32_t)h->C;
    out->tile_log2 = h->tile_log2;
    out->arena_capacity = h->capacity;
    out->host_store = h->host_store ? 1 : 0;
    return QS_OK;
}

// tf32 rounding of x (10 mantissa bits, to nearest, ties away from zero):
// the hi part of the 3xTF32 split of the gate operand.
static float tf32_round(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &b, 4);
    return r;
}

qs_status qs_apply_dense_gate(qs_state *h, const uint32_t *targets, uint32_t k, const double *matrix) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (!targets || !matrix) return fail(h, QS_ERR_ARG, "NULL argument");
    if (k < (uint32_t)qs::kMinDenseK || k > (uint32_t)qs::kMaxDenseK)
        return fail(h, QS_ERR_UNSUPPORTED_GATE, "dense gates act on 4 or 5 qubits (fused by optimize(block_size=k))");
    if (!h->staged_ok)
        return fail(h, QS_ERR_UNSUPPORTED_GATE, "dense k-qubit passes need HBM arenas (not the host store)");
    const int C = (int)h->C, n = (int)h->n, B = (int)h->B;
    if (n < qs::kDenseTileLog2) return fail(h, QS_ERR_ARG, "dense k-qubit passes need at least 12 qubits");
    for (uint32_t i = 0; i < k; ++i) {
        if (targets[i] >= h->n) return fail(h, QS_ERR_ARG, "gate target index out of range");
        for (uint32_t t = 0; t < i; ++t)
            if (targets[t] == targets[i]) return fail(h, QS_ERR_ARG, "duplicated qubit index in gate");
    }
    // tile: the chunk bits, the gate's qubits above them, padded with other
    // in-block qubits up to 2^12 amplitudes (every block of a tile then lies
    // in one group of this one-gate stage)
    const int jt = qs::kDenseTileLog2 - C;
    std::set<int> tq;
    for (uint32_t i = 0; i < k; ++i)
        if ((int)targets[i] >= C) tq.insert((int)targets[i]);
    if ((int)tq.size() > jt)
        return fail(h, QS_ERR_UNSUPPORTED_GATE, "a dense gate has more qubits above the chunk than a tile holds");
    for (int q = C; q < B && (int)tq.size() < jt; ++q) tq.insert(q);
    if ((int)tq.size() < jt) return fail(h, QS_ERR_ARG, "block too small for a dense k-qubit tile");
    const std::vector<int> tile(tq.begin(), tq.end());
    qs::DenseKGate dk{};
    dk.k = (int32_t)k;
    for (uint32_t i = 0; i < k; ++i) {
        const int q = (int)targets[i];
        dk.pos[i] = q < C ? q : C + (int)(std::find(tile.begin(), tile.end(), q) - tile.begin());
    }
    // the one-gate stage's groups: blocks differing only in the gate's
    // qubits at or above the block size (make_block_groups' rule)
    std::vector<uint32_t> b2g(h->nb);
    std::vector<int> outer;
    for (int q = B; q < n; ++q) {
        bool inner = false;
        for (uint32_t i = 0; i < k; ++i) inner = inner || (int)targets[i] == q;
        if (!inner) outer.push_back(q);
    }
    for (uint32_t b = 0; b < h->nb; ++b) {
        uint32_t gid = 0;
        for (size_t i = 0; i < outer.size(); ++i) gid |= ((b >> (outer[i] - B)) & 1u) << i;
        b2g[b] = gid;
    }
    const uint32_t ngroups = 1u << outer.size();
    // matrix operands
    const int K = 1 << k, Kp = 2 * K;
    std::vector<float> hi, lo;
    std::vector<double> mat;
    if (!h->f64) {
        hi.assign((size_t)Kp * Kp, 0.0f);
        lo.assign((size_t)Kp * Kp, 0.0f);
        for (int nrow = 0; nrow < Kp; ++nrow)
            for (int kc = 0; kc < Kp; ++kc) {
                const int r = nrow % K, c = kc % K;
                const double gr = matrix[2 * ((size_t)r * K + c)], gi = matrix[2 * ((size_t)r * K + c) + 1];
                // [[Gr, -Gi], [Gi, Gr]]: output rows Re y then Im y, input columns Re x then Im x
                const double v = nrow < K ? (kc < K ? gr : -gi) : (kc < K ? gi : gr);
                const float vh = tf32_round((float)v);
                const size_t off = qs::dense_k_operand_offset((uint32_t)nrow, (uint32_t)kc, (uint32_t)Kp) / 4;
                hi[off] = vh;
                lo[off] = tf32_round((float)v - vh);
            }
    } else {
        mat.assign(matrix, matrix + 2 * (size_t)K * K);
    }
    struct Tmp {
        std::vector<void *> p;
        ~Tmp() {
            for (void *q : p) cudaFree(q);
        }
    } tmp;
    cudaStream_t s = h->stream;
    uint32_t *db2g = nullptr;
    CUDA_TRY(h, cudaMalloc(&db2g, h->nb * sizeof(uint32_t)));
    tmp.p.push_back(db2g);
    CUDA_TRY(h, cudaMemcpyAsync(db2g, b2g.data(), h->nb * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    if (!h->f64) {
        float *d = nullptr;
        CUDA_TRY(h, cudaMalloc(&d, 2 * hi.size() * sizeof(float)));
        tmp.p.push_back(d);
        CUDA_TRY(h, cudaMemcpyAsync(d, hi.data(), hi.size() * 4, cudaMemcpyHostToDevice, s));
        CUDA_TRY(h, cudaMemcpyAsync(d + hi.size(), lo.data(), lo.size() * 4, cudaMemcpyHostToDevice, s));
        dk.bhi = d;
        dk.blo = d + hi.size();
    } else {
        double *d = nullptr;
        CUDA_TRY(h, cudaMalloc(&d, mat.size() * sizeof(double)));
        tmp.p.push_back(d);
        CUDA_TRY(h, cudaMemcpyAsync(d, mat.data(), mat.size() * 8, cudaMemcpyHostToDevice, s));
        dk.mat = d;
    }
    unsigned long long *dhist = nullptr;  // [0] stage total, [1] active blocks
    CUDA_TRY(h, cudaMalloc(&dhist, 2 * sizeof(unsigned long long)));
    tmp.p.push_back(dhist);
    CUDA_TRY(h, cudaMemsetAsync(dhist, 0, 2 * sizeof(unsigned long long), s));
    CUDA_TRY(h, cudaMemsetAsync(h->error_dev, 0, sizeof(int32_t), s));
    CUDA_TRY(h, cudaMemsetAsync(h->counters, 0, 8 * sizeof(unsigned long long), s));
    CUDA_TRY(h, qs::launch_stage_begin(db2g, h->mask, h->nb, h->group_active, ngroups, h->block_nz, h->block_acc,
                                       dhist + 1, s));
    const int out = h->cur ^ 1;
    qs::PassArgs a{};
    a.n = n;
    a.B = B;
    a.C = C;
    a.j = jt;
    for (int i = 0; i < jt; ++i) a.tq[i] = tile[i] - C;
    a.n_tiles = uint64_t(1) << (n - qs::kDenseTileLog2);
    a.rb = qs::kRegBits;
    a.codec = h->codec;
    a.meta_in = h->meta[h->mcur];
    a.arena_in = h->arena[h->cur];
    a.meta_out = h->meta[h->mcur ^ 1];
    a.arena_out = h->arena[out];
    a.perm = identity_perm();
    a.bump = h->counters + out;
    a.capacity = h->capacity;
    a.block_to_group = db2g;
    a.group_active = h->group_active;
    a.mask = h->mask;
    a.first_pass = 1;
    a.final_pass = 1;
    a.exact_zero = (h->flags & QS_FLAG_EXACT_ZERO_TEST) ? 1 : 0;
    a.header_batch = 4;
    a.block_nz = h->block_nz;
    a.block_bytes = h->block_acc;
    a.error = h->error_dev;
    a.stats = h->counters + 2;
    a.staged = 1;
    a.dense = dk;
    CUDA_TRY(h, cudaEventRecord(h->ev[0], s));
    CUDA_TRY(h, qs::launch_pass(h->f64, a, qs::kDenseTileLog2, s));
    CUDA_TRY(h, cudaEventRecord(h->ev[1], s));
    CUDA_TRY(h, qs::launch_stage_end(db2g, h->group_active, h->nb, h->block_nz, h->block_acc, h->mask,
                                     h->block_bytes, dhist, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    int32_t errflag = 0;
    unsigned long long ctr[8], hst[2];
    CUDA_TRY(h, cudaMemcpy(&errflag, h->error_dev, sizeof(errflag), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(ctr, h->counters, sizeof(ctr), cudaMemcpyDeviceToHost));
    CUDA_TRY(h, cudaMemcpy(hst, dhist, sizeof(hst), cudaMemcpyDeviceToHost));
    float ms = 0;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]));
    h->cur = out;
    h->mcur ^= 1;
    if (errflag == 2) return fail(h, QS_ERR_TIMEOUT, "a dense-gate pass gave up a bounded wait; the state is invalid");
    if (errflag) return fail(h, QS_ERR_CAPACITY, "compressed store overflowed its arena in a dense-gate pass");
    h->arena_used = ctr[out];
    h->history.push_back(hst[0]);
    h->st.bytes_read = ctr[2];
    h->st.bytes_written = ctr[3];
    h->st.tiles = ctr[4];
    h->st.kernel_ms = ms;
    h->st.apply_ms = ms;
    h->st.passes = 1;
    h->st.amp_gate_updates = hst[1] << h->B;
    return QS_OK;
}

qs_status qs_set_basis_state(qs_state *h, uint64_t basis) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (basis >> h->n) return fail(h, QS_ERR_ARG, "basis index out of range");
    return h->init_basis(basis);
}

qs_status qs_load_vector(qs_state *h, const double *vec) {
    if (!h || !vec) return fail(h, QS_ERR_ARG, "NULL argument");
    cudaStream_t s = h->stream;
    const uint64_t chunk_amps = uint64_t(1) << h->C;
    const uint64_t nslab = std::min<uint64_t>(std::max<uint64_t>(1, (uint64_t(1) << 24) / chunk_amps), h->nchunks);
    double *dbuf = nullptr;
    CUDA_TRY(h, cudaMalloc(&dbuf, nslab * chunk_amps * 2 * sizeof(double)));
    auto done = [&](qs_status st) { cudaFree(dbuf); return st; };
    if (cudaMemsetAsync(h->counters + h->cur, 0, sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(h->block_nz, 0, h->nb * sizeof(uint32_t), s) != cudaSuccess ||
        cudaMemsetAsync(h->block_acc, 0, h->nb * sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemsetAsync(h->error_dev, 0, sizeof(int32_t), s) != cudaSuccess)
        return done(fail(h, QS_ERR_CUDA, "memset failed"));
    for (uint64_t c0 = 0; c0 < h->nchunks; c0 += nslab) {
        const uint64_t cnt = std::min<uint64_t>(nslab, h->nchunks - c0);
        cudaError_t e = cudaMemcpyAsync(dbuf, vec + c0 * chunk_amps * 2, cnt * chunk_amps * 2 * sizeof(double),
                                        cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = qs::launch_encode(h->f64, dbuf, (int)h->B, (int)h->C, h->codec, c0, cnt, h->meta[h->mcur],
                                  h->arena[h->cur], h->counters + h->cur, h->capacity, h->block_nz, h->block_acc,
                                  h->error_dev, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return done(fail(h, QS_ERR_CUDA, std::string("load: ") + cudaGetErrorString(e)));
    }
    // mask = any non-zero in block; block bytes of zero blocks = 0
    std::vector<uint32_t> nz(h->nb);
    std::vector<unsigned long long> acc(h->nb);
    int32_t errflag = 0;
    unsigned long long used = 0;
    if (cudaMemcpy(nz.data(), h->block_nz, h->nb * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(acc.data(), h->block_acc, h->nb * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&errflag, h->error_dev, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&used, h->counters + h->cur, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return done(fail(h, QS_ERR_CUDA, "load readback failed"));
    if (errflag) return done(fail(h, QS_ERR_CAPACITY, "vector does not fit the arena"));
    std::vector<uint8_t> mk(h->nb);
    unsigned long long total = 0;
    for (uint32_t b = 0; b < h->nb; ++b) {
        mk[b] = nz[b] ? 1 : 0;
        if (!mk[b]) acc[b] = 0;
        total += acc[b];
    }
    if (cudaMemcpy(h->mask, mk.data(), h->nb, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->block_bytes, acc.data(), h->nb * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        return done(fail(h, QS_ERR_CUDA, "load upload failed"));
    h->arena_used = used;
    h->history.assign(1, total);
    return done(QS_OK);
}

// ---- Pauli expectation values
// Terms are batched so that each batch's flip qubits at or above the chunk
// size fit in one tile; each batch is one read-only pass.
static bool same_geometry(const qs_state *a, const qs_state *b) {
    return a->n == b->n && a->B == b->B && a->C == b->C && a->f64 == b->f64 && a->codec.m == b->codec.m &&
           a->codec.L == b->codec.L;
}

// Pauli sums over the ket store h, with bra store `bra` (NULL: the ket).
static qs_status pauli_sums(qs_state *h, const qs_state *bra, const uint64_t *x_masks, const uint64_t *z_masks,
                            size_t nterms, double *out);

qs_status qs_expectation_pauli(qs_state *h, const uint64_t *x_masks, const uint64_t *z_masks, size_t nterms,
                               double *out) {
    return pauli_sums(h, nullptr, x_masks, z_masks, nterms, out);
}

qs_status qs_transition_pauli(const qs_state *bra, qs_state *ket, const uint64_t *x_masks, const uint64_t *z_masks,
                              size_t nterms, double *out) {
    if (!bra || !ket) return fail(ket, QS_ERR_ARG, "NULL handle");
    if (!same_geometry(bra, ket)) return fail(ket, QS_ERR_ARG, "bra and ket differ in qubits, block, chunk, dtype or codec");
    if (bra->stream != ket->stream) CUDA_TRY(ket, cudaStreamSynchronize(bra->stream));
    return pauli_sums(ket, bra, x_masks, z_masks, nterms, out);
}

static qs_status pauli_sums(qs_state *h, const qs_state *bra, const uint64_t *x_masks, const uint64_t *z_masks,
                            size_t nterms, double *out) {
    if (!h || (nterms && (!x_masks || !z_masks || !out))) return fail(h, QS_ERR_ARG, "NULL argument");
    const int C = (int)h->C;
    const int jmax = std::min(h->tile_log2 - C, qs::kMaxTileQubits);
    const uint64_t full = h->n >= 64 ? ~0ull : ((1ull << h->n) - 1);
    for (size_t t = 0; t < nterms; ++t) {
        if ((x_masks[t] | z_masks[t]) & ~full) return fail(h, QS_ERR_ARG, "Pauli term acts outside the register");
        int hi = 0;
        for (int q = C; q < (int)h->n; ++q) hi += (x_masks[t] >> q) & 1;
        if (hi > jmax) return fail(h, QS_ERR_ARG, "Pauli term flips more qubits than a tile holds");
    }
    // greedy batches
    std::vector<std::vector<size_t>> batches;
    std::vector<std::set<int>> tiles;
    for (size_t t = 0; t < nterms; ++t) {
        std::set<int> need;
        for (int q = C; q < (int)h->n; ++q)
            if ((x_masks[t] >> q) & 1) need.insert(q);
        bool placed = false;
        for (size_t b = 0; b < batches.size() && !placed; ++b) {
            std::set<int> u = tiles[b];
            u.insert(need.begin(), need.end());
            if ((int)u.size() <= jmax && batches[b].size() < 256) {
                tiles[b] = u;
                batches[b].push_back(t);
                placed = true;
            }
        }
        if (!placed) {
            batches.push_back({t});
            tiles.push_back(need);
        }
    }
    double *dout = nullptr;
    qs::PauliTerm *dterms = nullptr;
    qs_status rs = QS_OK;
    cudaError_t e = cudaMalloc(&dout, std::max<size_t>(1, 2 * nterms) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dterms, std::max<size_t>(1, nterms) * sizeof(qs::PauliTerm));
    if (e == cudaSuccess) e = cudaMemsetAsync(dout, 0, std::max<size_t>(1, 2 * nterms) * sizeof(double), h->stream);
    std::vector<qs::PauliTerm> host(nterms);
    for (size_t b = 0; b < batches.size() && e == cudaSuccess; ++b) {
        std::set<int> tq = tiles[b];
        for (int q = C; q < (int)h->n && (int)tq.size() < std::min(3, jmax); ++q) tq.insert(q);
        std::vector<int> tv(tq.begin(), tq.end());
        auto local = [&](uint64_t m, uint64_t *outside) {
            uint32_t r = 0;
            uint64_t o = 0;
            for (int q = 0; q < (int)h->n; ++q) {
                if (!((m >> q) & 1)) continue;
                if (q < C) r |= 1u << q;
                else {
                    auto it = std::find(tv.begin(), tv.end(), q);
                    if (it != tv.end()) r |= 1u << (C + (int)(it - tv.begin()));
                    else o |= 1ull << q;
                }
            }
            if (outside) *outside = o;
            return r;
        };
        std::vector<qs::PauliTerm> bt;
        for (size_t t : batches[b]) {
            qs::PauliTerm pt{};
            uint64_t dummy = 0;
            pt.xt = local(x_masks[t], &dummy);
            pt.zt = local(z_masks[t], &pt.zo);
            pt.xg = x_masks[t];
            pt.zg = z_masks[t];
            bt.push_back(pt);
        }
        // the batch's terms are laid out contiguously in dterms at offset of the first
        const size_t off = batches[b][0];
        (void)off;
        qs::PauliTerm *bdev = nullptr;
        double *bout = nullptr;
        e = cudaMalloc(&bdev, bt.size() * sizeof(qs::PauliTerm));
        if (e == cudaSuccess) e = cudaMalloc(&bout, 2 * bt.size() * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpyAsync(bdev, bt.data(), bt.size() * sizeof(qs::PauliTerm), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(bout, 0, 2 * bt.size() * sizeof(double), h->stream);
        if (e == cudaSuccess) {
            qs::ExpectArgs a{};
            a.n = (int)h->n;
            a.B = (int)h->B;
            a.C = C;
            a.j = (int)tv.size();
            for (int k = 0; k < a.j; ++k) a.tq[k] = tv[k] - C;
            a.n_tiles = uint64_t(1) << (h->n - C - a.j);
            a.meta = h->meta[h->mcur];
            a.arena = h->arena[h->cur];
            a.mask = h->mask;
            a.codec = h->codec;
            a.terms = bdev;
            a.nterms = (int)bt.size();
            a.out = bout;
            if (bra) {
                a.meta_bra = bra->meta[bra->mcur];
                a.arena_bra = bra->arena[bra->cur];
                a.mask_bra = bra->mask;
            }
            e = qs::launch_expect(h->f64, a, h->stream);
        }
        std::vector<double> hb(2 * bt.size());
        if (e == cudaSuccess) e = cudaMemcpyAsync(hb.data(), bout, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e == cudaSuccess)
            for (size_t k = 0; k < batches[b].size(); ++k) {
                out[2 * batches[b][k]] = hb[2 * k];
                out[2 * batches[b][k] + 1] = hb[2 * k + 1];
            }
        if (bdev) cudaFree(bdev);
        if (bout) cudaFree(bout);
    }
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        rs = fail(h, QS_ERR_CUDA, std::string("expectation: ") + cudaGetErrorString(e));
    }
    if (dout) cudaFree(dout);
    if (dterms) cudaFree(dterms);
    return rs;
}

// ---- out := (sum_t c_t Z^{z_t}) in, one tile pass from in's store into out's
qs_status qs_apply_diagonal_pauli_sum(qs_state *out, const qs_state *in, const uint64_t *z_masks,
                                      const double *coefs, size_t nterms) {
    if (!out || !in) return fail(out, QS_ERR_ARG, "NULL handle");
    if (out == in) return fail(out, QS_ERR_ARG, "out and in must be different states");
    if (nterms && (!z_masks || !coefs)) return fail(out, QS_ERR_ARG, "NULL argument");
    if (nterms > (size_t)qs::kMaxDiagTerms)
        return fail(out, QS_ERR_ARG, "at most " + std::to_string(qs::kMaxDiagTerms) + " terms");
    if (!same_geometry(out, in)) return fail(out, QS_ERR_ARG, "in and out differ in qubits, block, chunk, dtype or codec");
    const uint64_t full = out->n >= 64 ? ~0ull : ((1ull << out->n) - 1);
    for (size_t t = 0; t < nterms; ++t)
        if (z_masks[t] & ~full) return fail(out, QS_ERR_ARG, "Pauli term acts outside the register");
    if (in->stream != out->stream) CUDA_TRY(out, cudaStreamSynchronize(in->stream));
    cudaStream_t s = out->stream;
    const int C = (int)out->C;
    const int jmax = std::min(out->tile_log2 - C, qs::kMaxTileQubits);
    const int j = std::max(0, std::min<int>({jmax, 3, (int)out->n - C}));
    std::vector<int> tv;
    for (int q = C; q < C + j; ++q) tv.push_back(q);
    if (C + j < qs::kRegBits) return fail(out, QS_ERR_ARG, "state too small for a tile pass");
    std::vector<qs::PauliTerm> terms(nterms);
    for (size_t t = 0; t < nterms; ++t) {
        qs::PauliTerm pt{};
        for (int q = 0; q < (int)out->n; ++q) {
            if (!((z_masks[t] >> q) & 1)) continue;
            if (q < C + j) pt.zt |= 1u << q;  // tile qubits are the lowest C + j
            else pt.zo |= 1ull << q;
        }
        pt.zg = z_masks[t];
        terms[t] = pt;
    }
    qs::PauliTerm *dterms = nullptr;
    double *dcoef = nullptr;
    uint32_t *ident = nullptr;
    auto cleanup = [&]() {
        if (dterms) cudaFree(dterms);
        if (dcoef) cudaFree(dcoef);
        if (ident) cudaFree(ident);
    };
    cudaError_t e = cudaMalloc(&dterms, std::max<size_t>(1, nterms) * sizeof(qs::PauliTerm));
    if (e == cudaSuccess) e = cudaMalloc(&dcoef, std::max<size_t>(1, 2 * nterms) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ident, out->nb * sizeof(uint32_t));
    std::vector<uint32_t> hid(out->nb);
    for (uint32_t b = 0; b < out->nb; ++b) hid[b] = b;
    if (e == cudaSuccess && nterms)
        e = cudaMemcpyAsync(dterms, terms.data(), nterms * sizeof(qs::PauliTerm), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && nterms)
        e = cudaMemcpyAsync(dcoef, coefs, 2 * nterms * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ident, hid.data(), hid.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    const int o = out->cur ^ 1;
    if (e == cudaSuccess) e = cudaMemsetAsync(out->counters, 0, 8 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(out->error_dev, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(out->block_nz, 0, out->nb * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(out->block_acc, 0, out->nb * sizeof(unsigned long long), s);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        cleanup();
        return fail(out, QS_ERR_CUDA, std::string("diagonal Pauli sum: ") + cudaGetErrorString(e));
    }
    qs::PassArgs a{};
    a.header_batch = 4;
    a.n = (int)out->n;
    a.B = (int)out->B;
    a.C = C;
    a.j = j;
    for (int k = 0; k < j; ++k) a.tq[k] = tv[k] - C;
    a.n_tiles = uint64_t(1) << (out->n - C - j);
    a.nsweeps = 0;
    a.rb = qs::kRegBits;
    a.codec = out->codec;
    a.meta_in = in->meta[in->mcur];
    a.arena_in = in->arena[in->cur];
    a.meta_out = out->meta[out->mcur ^ 1];
    a.arena_out = out->arena[o];
    a.bump = out->counters + o;
    a.capacity = out->capacity;
    a.block_to_group = ident;
    a.group_active = in->mask;  // stored blocks of `in` are processed, the others stay zero
    a.mask = in->mask;
    a.first_pass = 1;
    a.final_pass = 1;
    a.exact_zero = (out->flags & QS_FLAG_EXACT_ZERO_TEST) ? 1 : 0;
    a.block_nz = out->block_nz;
    a.block_bytes = out->block_acc;
    a.error = out->error_dev;
    a.stats = out->counters + 2;
    a.perm = identity_perm();
    a.diag.terms = dterms;
    a.diag.coefs = dcoef;
    a.diag.nterms = (int)nterms;
    e = qs::launch_pass(out->f64, a, out->tile_log2, s);
    // out keeps in's zero-block mask; its block bytes are the new ones
    if (e == cudaSuccess) e = cudaMemcpyAsync(out->mask, in->mask, out->nb, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
        e = qs::launch_stage_end(ident, in->mask, out->nb, out->block_nz, out->block_acc, out->mask, out->block_bytes,
                                 out->counters + 7, s);  // counters were zeroed above
    int32_t errflag = 0;
    unsigned long long ctr[8] = {0}, total = 0;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpy(&errflag, out->error_dev, sizeof(errflag), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(ctr, out->counters, sizeof(ctr), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) total = ctr[7];
    cleanup();
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(out, QS_ERR_CUDA, std::string("diagonal Pauli sum: ") + cudaGetErrorString(e));
    }
    if (errflag)
        return fail(out, QS_ERR_CAPACITY, "compressed store overflowed its arena; the state is invalid");
    out->cur = o;
    out->mcur ^= 1;
    out->arena_used = ctr[o];
    out->history.assign(1, total);
    return QS_OK;
}

// ---- passes over two compressed stores (the compressed adjoint)
// One launch of dual_pass_kernel over A and B with the tile qubits `tile`;
// ops and sums already on the device.  Written stores switch to their other
// arena; afterwards every block of a written store is stored.
// Register sweeps of a two-store launch (device pointers; see DualPassArgs).
struct DualSweepRef {
    const qs::Sweep *sweeps = nullptr;
    int nsweeps = 0, rb = 0;
    const qs::ROp *rops = nullptr;
    const void *pool = nullptr;
    const std::vector<int> *outer = nullptr;
};

static qs_status dual_launch(qs_state *A, qs_state *B, const std::vector<int> &tile, const qs::DualOp *ops,
                             int nops, bool write_a, bool b_zero, double *sums, int nslots,
                             const DualSweepRef *sw = nullptr) {
    cudaStream_t s = A->stream;
    const int C = (int)A->C;
    qs::DualPassArgs d{};
    if (sw && sw->nsweeps > 0) {
        d.sweeps = sw->sweeps;
        d.nsweeps = sw->nsweeps;
        d.rb = sw->rb;
        d.rops = sw->rops;
        d.pool = sw->pool;
        d.nouter = (int32_t)sw->outer->size();
        for (int i = 0; i < d.nouter; ++i) d.outer_q[i] = (int8_t)(*sw->outer)[i];
    }
    d.n = (int)A->n;
    d.B = (int)A->B;
    d.C = C;
    d.j = (int)tile.size();
    for (int k = 0; k < d.j; ++k) d.tq[k] = tile[k] - C;
    d.n_tiles = uint64_t(1) << (A->n - C - d.j);
    d.ops = ops;
    d.nops = nops;
    d.codec = A->codec;
    d.sums = sums;
    d.nslots = nslots;
    d.error = A->error_dev;
    auto store = [&](qs_state *h, bool zero_in, bool write) {
        qs::DualStore st{};
        st.meta_in = zero_in ? nullptr : h->meta[h->mcur];
        st.arena_in = h->arena[h->cur];
        st.mask_in = h->mask;
        st.meta_out = write ? h->meta[h->mcur ^ 1] : nullptr;
        st.arena_out = h->arena[h->cur ^ 1];
        st.bump = h->counters + (h->cur ^ 1);
        st.capacity = h->capacity;
        st.block_bytes = h->block_acc;
        return st;
    };
    d.a = store(A, false, write_a);
    d.b = store(B, b_zero, true);
    for (qs_state *h : {A, B}) {
        if (h == A && !write_a) continue;
        CUDA_TRY(h, cudaMemsetAsync(h->counters + (h->cur ^ 1), 0, sizeof(unsigned long long), s));
        CUDA_TRY(h, cudaMemsetAsync(h->block_acc, 0, h->nb * sizeof(unsigned long long), s));
    }
    CUDA_TRY(A, qs::launch_dual_pass(A->f64, d, s));
    for (qs_state *h : {A, B}) {
        if (h == A && !write_a) continue;
        h->cur ^= 1;
        h->mcur ^= 1;
        CUDA_TRY(h, cudaMemsetAsync(h->mask, 1, h->nb, s));
        CUDA_TRY(h, cudaMemcpyAsync(h->block_bytes, h->block_acc, h->nb * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToDevice, s));
    }
    return QS_OK;
}

// After a series of dual passes: check the error flag, record the arenas'
// use and the stores' totals.
static qs_status dual_finish(qs_state *A, qs_state *B, bool wrote_a) {
    CUDA_TRY(A, cudaStreamSynchronize(A->stream));
    int32_t errflag = 0;
    CUDA_TRY(A, cudaMemcpy(&errflag, A->error_dev, sizeof(errflag), cudaMemcpyDeviceToHost));
    if (errflag)
        return fail(A, QS_ERR_CAPACITY, "a compressed store overflowed its arena in a two-store pass; set "
                                        "QOMPSIM_ARENA_BYTES larger");
    for (qs_state *h : {A, B}) {
        if (h == A && !wrote_a) continue;
        unsigned long long used = 0;
        CUDA_TRY(h, cudaMemcpy(&used, h->counters + h->cur, sizeof(used), cudaMemcpyDeviceToHost));
        h->arena_used = used;
        h->history.assign(1, used + h->nchunks * sizeof(qs::ChunkMeta));
    }
    return QS_OK;
}

// Tile-local masks of a Pauli string for tile qubits `tile` (flip qubits
// must lie in the tile).
static qs::PauliTerm tile_term(uint64_t xm, uint64_t zm, const std::vector<int> &tile, int C, int n) {
    qs::PauliTerm t{};
    for (int q = 0; q < n; ++q) {
        int tp = q < C ? q : -1;
        if (q >= C) {
            auto it = std::find(tile.begin(), tile.end(), q);
            if (it != tile.end()) tp = C + (int)(it - tile.begin());
        }
        if ((xm >> q) & 1) t.xt |= 1u << tp;
        if ((zm >> q) & 1) {
            if (tp >= 0) t.zt |= 1u << tp;
            else t.zo |= 1ull << q;
        }
    }
    t.xg = xm;
    t.zg = zm;
    return t;
}

static qs_status dual_check(qs_state *A, const qs_state *B) {
    if (!same_geometry(A, B)) return fail(A, QS_ERR_ARG, "the two states differ in qubits, block, chunk, dtype or codec");
    if (A->stream != B->stream) return fail(A, QS_ERR_ARG, "the two states must share a stream");
    if (A->host_store || B->host_store) return fail(A, QS_ERR_ARG, "two-store passes need HBM arenas");
    if (A->C + std::min<int>(4, (int)A->n - (int)A->C) < qs::kRegBits)
        return fail(A, QS_ERR_ARG, "state too small for a two-store pass");
    return QS_OK;
}

// Tiles of the two-store passes: 2^12 amplitudes (two value tiles of 64 KB
// in complex128, 32 KB in complex64); QOMPSIM_DUAL_TILE_LOG2 = 13 doubles
// them (complex64 only), halving the passes of a gate sequence's qubits.
static int dual_tile_log2(const qs_state *h) {
    const int t = env_int("QOMPSIM_DUAL_TILE_LOG2", 12);
    return (t == 13 && !h->f64) ? 13 : 12;
}

qs_status qs_apply_pauli_sum(qs_state *out, qs_state *in, const uint64_t *x_masks, const uint64_t *z_masks,
                             const double *coefs, size_t nterms) {
    if (!out || !in) return fail(out, QS_ERR_ARG, "NULL handle");
    if (out == in) return fail(out, QS_ERR_ARG, "out and in must be different states");
    if (nterms && (!x_masks || !z_masks || !coefs)) return fail(out, QS_ERR_ARG, "NULL argument");
    qs_status st = dual_check(in, out);
    if (st != QS_OK) return fail(out, st, in->err);
    const int C = (int)out->C, n = (int)out->n;
    const uint64_t full = n >= 64 ? ~0ull : ((1ull << n) - 1);
    for (size_t t = 0; t < nterms; ++t)
        if ((x_masks[t] | z_masks[t]) & ~full) return fail(out, QS_ERR_ARG, "Pauli term acts outside the register");
    const int jmax = std::min(dual_tile_log2(in) - C, n - C);
    // terms in order, grouped so that each group's flip qubits >= C fit a tile
    std::vector<std::vector<size_t>> groups;
    std::vector<std::set<int>> gq;
    for (size_t t = 0; t < nterms; ++t) {
        std::set<int> q;
        for (int b = C; b < n; ++b)
            if ((x_masks[t] >> b) & 1) q.insert(b);
        if ((int)q.size() > jmax) return fail(out, QS_ERR_ARG, "a Pauli term flips more qubits than a tile holds");
        bool placed = false;
        for (size_t g = 0; g < groups.size() && !placed; ++g) {
            std::set<int> u = gq[g];
            u.insert(q.begin(), q.end());
            if ((int)u.size() <= jmax) {
                gq[g] = u;
                groups[g].push_back(t);
                placed = true;
            }
        }
        if (!placed) {
            groups.push_back({t});
            gq.push_back(q);
        }
    }
    if (groups.empty()) groups.push_back({});
    std::vector<qs::DualOp> ops;
    std::vector<std::vector<int>> tiles;
    std::vector<size_t> op_off;
    for (size_t g = 0; g < groups.size(); ++g) {
        std::set<int> tq = g < gq.size() ? gq[g] : std::set<int>();
        for (int q = C; q < n && (int)tq.size() < jmax; ++q) tq.insert(q);
        std::vector<int> tile(tq.begin(), tq.end());
        tiles.push_back(tile);
        op_off.push_back(ops.size());
        for (size_t t : groups[g]) {
            qs::DualOp o{};
            o.kind = qs::DOP_ACCUM;
            o.term = tile_term(x_masks[t], z_masks[t], tile, C, n);
            o.coef[0] = coefs[2 * t];
            o.coef[1] = coefs[2 * t + 1];
            ops.push_back(o);
        }
    }
    op_off.push_back(ops.size());
    qs::DualOp *dops = nullptr;
    CUDA_TRY(out, cudaMalloc(&dops, std::max<size_t>(1, ops.size()) * sizeof(qs::DualOp)));
    struct Free { void *p; ~Free() { if (p) cudaFree(p); } } fr{dops};
    if (!ops.empty())
        CUDA_TRY(out, cudaMemcpyAsync(dops, ops.data(), ops.size() * sizeof(qs::DualOp), cudaMemcpyHostToDevice,
                                      out->stream));
    CUDA_TRY(out, cudaMemsetAsync(in->error_dev, 0, sizeof(int32_t), out->stream));
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CUDA_TRY(out, cudaEventCreate(&ev0));
    struct EvFree { cudaEvent_t &a, &b; ~EvFree() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); } } evf{ev0, ev1};
    CUDA_TRY(out, cudaEventCreate(&ev1));
    CUDA_TRY(out, cudaEventRecord(ev0, out->stream));
    for (size_t g = 0; g < tiles.size(); ++g) {
        st = dual_launch(in, out, tiles[g], dops + op_off[g], (int)(op_off[g + 1] - op_off[g]), false, g == 0,
                         nullptr, 0);
        if (st != QS_OK) return fail(out, st, in->err);
    }
    CUDA_TRY(out, cudaEventRecord(ev1, out->stream));
    st = dual_finish(in, out, false);
    if (st != QS_OK) return fail(out, st, in->err);
    {
        float pm = 0.f;
        if (cudaEventElapsedTime(&pm, ev0, ev1) == cudaSuccess) out->st.pair_ms = pm;
    }
    return QS_OK;
}

qs_status qs_adjoint(qs_state *psi, qs_state *lam, const qs_gate *gates, const int32_t *slots, const uint64_t *gen_x,
                     const uint64_t *gen_z, size_t count, double *out, uint32_t nslots) {
    if (!psi || !lam || (count && (!gates || !slots || !gen_x || !gen_z)) || (nslots && !out))
        return fail(psi, QS_ERR_ARG, "NULL argument");
    if (psi == lam) return fail(psi, QS_ERR_ARG, "psi and lam must be distinct states");
    qs_status st = dual_check(psi, lam);
    if (st != QS_OK) return st;
    for (size_t i = 0; i < count; ++i)
        if (slots[i] >= (int32_t)nslots) return fail(psi, QS_ERR_ARG, "slot index out of range");
    const int C = (int)psi->C, n = (int)psi->n;
    std::vector<CGate> cg(count);
    for (size_t i = 0; i < count; ++i) {
        std::string e;
        if (!canonicalize(gates[i], false, psi->n, &cg[i], &e))
            return fail(psi, QS_ERR_UNSUPPORTED_GATE, "gate " + std::to_string(i) + ": " + e);
    }
    // generators' flip qubits must lie in the tile too: treat them as mixing
    for (size_t i = 0; i < count; ++i) {
        if (slots[i] < 0) continue;
        uint64_t covered = 0;
        for (int b = 0; b < cg[i].nq; ++b) {
            covered |= 1ull << cg[i].q[b];
            if ((gen_x[i] >> cg[i].q[b]) & 1) cg[i].mix[b] = true;
        }
        if (gen_x[i] & ~covered) return fail(psi, QS_ERR_ARG, "a generator flips a qubit its gate does not act on");
    }
    const int jmax = std::min(dual_tile_log2(psi) - C, n - C);
    std::vector<uint32_t> ids(count);
    for (size_t i = 0; i < count; ++i) ids[i] = (uint32_t)i;
    // Commuting gates may change places here too: a gate G moved across the
    // derivative sum of gate k commutes with U_k, so it shares with U_k only
    // qubits on which neither mixes, and there P_k is I or Z (its flip qubits
    // count as mixing qubits of gate k above); then G commutes with P_k and
    // <G^-1 lam| P_k |G^-1 psi> = <lam| P_k |psi>.
    auto pl = env_int("QOMPSIM_DAG_PLAN", 1) ? plan_passes_dag(ids, cg, C, jmax, jmax, C, n)
                                             : plan_passes(ids, cg, C, jmax, jmax, C, n);
    // launches: a pass's gates, split so that each launch has at most
    // kMaxDualSlots derivative sums
    struct Launch {
        std::vector<int> tile;
        size_t op_off, nops, out_off;
        std::vector<int32_t> local_to_global;
        std::vector<uint32_t> gates;
        // register sweeps over both stores (fused = false: one shared-memory
        // sweep per DualOp instead)
        bool fused = false;
        size_t sw_off = 0, nsw = 0, rop_off = 0;
        std::vector<int> outer;
    };
    std::vector<qs::DualOp> ops;
    std::vector<Launch> launches;
    size_t nout = 0;
    for (auto &p : pl) {
        for (size_t g0 = 0; g0 < p.gates.size();) {
            Launch L{};
            L.tile = p.tile;
            L.op_off = ops.size();
            L.out_off = nout;
            size_t g1 = g0;
            for (; g1 < p.gates.size(); ++g1) {
                const uint32_t gi = p.gates[g1];
                if (slots[gi] >= 0) {
                    if (L.local_to_global.size() >= (size_t)qs::kMaxDualSlots) break;
                    qs::DualOp o{};
                    o.kind = qs::DOP_SUM;
                    o.slot = (int32_t)L.local_to_global.size();
                    o.term = tile_term(gen_x[gi], gen_z[gi], p.tile, C, n);
                    ops.push_back(o);
                    L.local_to_global.push_back(slots[gi]);
                }
                qs::DualOp o{};
                o.kind = qs::DOP_GATE_AB;
                o.g = to_kgate(cg[gi], p.tile, C);
                ops.push_back(o);
                L.gates.push_back(gi);
            }
            L.nops = ops.size() - L.op_off;
            nout += L.local_to_global.size();
            launches.push_back(std::move(L));
            g0 = g1;
        }
    }
    // Register sweeps for every launch: the launch's gates in order, each
    // parametric gate's derivative sum placed just before it (a pseudo-gate
    // with the gate's qubits and mixing bits, so that the two share a sweep
    // and the generator's flip qubits are register bits).
    const int RB = psi->f64 ? qs::kDualRegBitsF64 : qs::kDualRegBitsF32;
    std::vector<qs::Sweep> all_sw;
    std::vector<qs::ROp> all_rops;
    std::vector<cplx> all_pool;
    if (env_int("QOMPSIM_DUAL_SWEEPS", 1)) {
        for (Launch &L : launches) {
            DualSweepPlan dp;
            if (!plan_dual_sweeps(cg, L.gates, slots, gen_x, gen_z, L.tile, C, RB, &all_sw, &all_rops, &all_pool, &dp))
                continue;
            L.fused = true;
            L.sw_off = dp.sw_off;
            L.nsw = dp.nsw;
            L.rop_off = dp.rop_off;
            L.outer = dp.outer;
        }
    }
    qs::DualOp *dops = nullptr;
    double *dsum = nullptr;
    CUDA_TRY(psi, cudaMalloc(&dops, std::max<size_t>(1, ops.size()) * sizeof(qs::DualOp)));
    struct Free { void *p; ~Free() { if (p) cudaFree(p); } } f1{dops};
    CUDA_TRY(psi, cudaMalloc(&dsum, std::max<size_t>(1, 2 * nout) * sizeof(double)));
    Free f2{dsum};
    cudaStream_t s = psi->stream;
    qs::Sweep *dsw = nullptr;
    qs::ROp *drops = nullptr;
    void *dpool = nullptr;
    const size_t pool_bytes = all_pool.size() * (psi->f64 ? 16 : 8);
    CUDA_TRY(psi, cudaMalloc(&dsw, std::max<size_t>(1, all_sw.size()) * sizeof(qs::Sweep)));
    Free f3{dsw};
    CUDA_TRY(psi, cudaMalloc(&drops, std::max<size_t>(1, all_rops.size()) * sizeof(qs::ROp)));
    Free f4{drops};
    CUDA_TRY(psi, cudaMalloc(&dpool, std::max<size_t>(16, pool_bytes)));
    Free f5{dpool};
    std::vector<float> pool_f;
    std::vector<double> pool_d;
    if (psi->f64) pool_d = pool_as<double>(all_pool);
    else pool_f = pool_as<float>(all_pool);
    if (!all_sw.empty())
        CUDA_TRY(psi, cudaMemcpyAsync(dsw, all_sw.data(), all_sw.size() * sizeof(qs::Sweep), cudaMemcpyHostToDevice, s));
    if (!all_rops.empty())
        CUDA_TRY(psi, cudaMemcpyAsync(drops, all_rops.data(), all_rops.size() * sizeof(qs::ROp), cudaMemcpyHostToDevice,
                                      s));
    if (pool_bytes)
        CUDA_TRY(psi, cudaMemcpyAsync(dpool, psi->f64 ? (const void *)pool_d.data() : (const void *)pool_f.data(),
                                      pool_bytes, cudaMemcpyHostToDevice, s));
    if (!ops.empty())
        CUDA_TRY(psi, cudaMemcpyAsync(dops, ops.data(), ops.size() * sizeof(qs::DualOp), cudaMemcpyHostToDevice, s));
    CUDA_TRY(psi, cudaMemsetAsync(dsum, 0, std::max<size_t>(1, 2 * nout) * sizeof(double), s));
    CUDA_TRY(psi, cudaMemsetAsync(psi->error_dev, 0, sizeof(int32_t), s));
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CUDA_TRY(psi, cudaEventCreate(&ev0));
    struct EvFree { cudaEvent_t &a, &b; ~EvFree() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); } } evf{ev0, ev1};
    CUDA_TRY(psi, cudaEventCreate(&ev1));
    CUDA_TRY(psi, cudaEventRecord(ev0, s));
    for (const Launch &L : launches) {
        DualSweepRef ref{};
        if (L.fused) {
            ref.sweeps = dsw + L.sw_off;
            ref.nsweeps = (int)L.nsw;
            ref.rb = RB;
            ref.rops = drops + L.rop_off;
            ref.pool = dpool;
            ref.outer = &L.outer;
        }
        st = dual_launch(psi, lam, L.tile, dops + L.op_off, (int)L.nops, true, false, dsum + 2 * L.out_off,
                         (int)L.local_to_global.size(), L.fused ? &ref : nullptr);
        if (st != QS_OK) return st;
    }
    CUDA_TRY(psi, cudaEventRecord(ev1, s));
    std::vector<double> h(2 * nout);
    if (nout) CUDA_TRY(psi, cudaMemcpyAsync(h.data(), dsum, 2 * nout * sizeof(double), cudaMemcpyDeviceToHost, s));
    st = dual_finish(psi, lam, true);
    {
        float pm = 0.f;
        if (cudaEventElapsedTime(&pm, ev0, ev1) == cudaSuccess) psi->st.pair_ms = pm;
    }
    if (st != QS_OK) return st;
    std::vector<double> acc(2 * (size_t)nslots, 0.0);
    for (const Launch &L : launches)
        for (size_t k = 0; k < L.local_to_global.size(); ++k) {
            acc[2 * L.local_to_global[k]] += h[2 * (L.out_off + k)];
            acc[2 * L.local_to_global[k] + 1] += h[2 * (L.out_off + k) + 1];
        }
    for (size_t i = 0; i < acc.size(); ++i) out[i] = acc[i];
    return QS_OK;
}

// ---- device checkpoints of the compressed store
qs_status qs_checkpoint(qs_state *h, uint32_t slot) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (slot >= 64) return fail(h, QS_ERR_ARG, "checkpoint slot must be < 64");
    if (h->ckpt.size() <= slot) h->ckpt.resize(slot + 1);
    auto &c = h->ckpt[slot];
    const uint64_t meta_bytes = h->nchunks * sizeof(qs::ChunkMeta);
    if (!c.meta) {
        CUDA_TRY(h, cudaMalloc(&c.meta, meta_bytes));
        CUDA_TRY(h, cudaMalloc(&c.mask, h->nb));
        CUDA_TRY(h, cudaMalloc(&c.block_bytes, h->nb * sizeof(unsigned long long)));
    }
    if (c.arena_cap < h->arena_used) {
        if (c.arena) cudaFree(c.arena);
        c.arena = nullptr;
        c.arena_cap = 0;
        const uint64_t cap = std::max<uint64_t>(128, (h->arena_used + 127) / 128 * 128);
        cudaError_t e = cudaMalloc(&c.arena, cap);
        if (e != cudaSuccess)
            return fail(h, e == cudaErrorMemoryAllocation ? QS_ERR_CAPACITY : QS_ERR_CUDA,
                        std::string("checkpoint: ") + cudaGetErrorString(e));
        c.arena_cap = cap;
    }
    cudaStream_t s = h->stream;
    CUDA_TRY(h, cudaMemcpyAsync(c.meta, h->meta[h->mcur], meta_bytes, cudaMemcpyDeviceToDevice, s));
    if (h->arena_used)
        CUDA_TRY(h, cudaMemcpyAsync(c.arena, h->arena[h->cur], h->arena_used, cudaMemcpyDefault, s));
    CUDA_TRY(h, cudaMemcpyAsync(c.mask, h->mask, h->nb, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(h, cudaMemcpyAsync(c.block_bytes, h->block_bytes, h->nb * sizeof(unsigned long long),
                                cudaMemcpyDeviceToDevice, s));
    c.used = h->arena_used;
    c.history = h->history;
    return QS_OK;
}

qs_status qs_restore(qs_state *h, uint32_t slot) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (slot >= h->ckpt.size() || !h->ckpt[slot].meta) return fail(h, QS_ERR_STATE, "no checkpoint in this slot");
    auto &c = h->ckpt[slot];
    cudaStream_t s = h->stream;
    CUDA_TRY(h, cudaMemcpyAsync(h->meta[h->mcur], c.meta, h->nchunks * sizeof(qs::ChunkMeta), cudaMemcpyDeviceToDevice, s));
    if (c.used) CUDA_TRY(h, cudaMemcpyAsync(h->arena[h->cur], c.arena, c.used, cudaMemcpyDefault, s));
    CUDA_TRY(h, cudaMemcpyAsync(h->mask, c.mask, h->nb, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(h, cudaMemcpyAsync(h->block_bytes, c.block_bytes, h->nb * sizeof(unsigned long long),
                                cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    h->arena_used = c.used;
    h->history = c.history;
    return QS_OK;
}

qs_status qs_free_checkpoint(qs_state *h, uint32_t slot) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    if (slot < h->ckpt.size()) qs_state::free_checkpoint(h->ckpt[slot]);
    return QS_OK;
}

// ---- store serialisation
struct StoreHeader {
    char magic[8];
    uint32_t n, B, C, f64;
    int32_t m, L;
    uint64_t nb, nchunks, arena_bytes;
};

qs_status qs_export_store(qs_state *h, void *buf, uint64_t cap, uint64_t *size) {
    if (!h || !size) return fail(h, QS_ERR_ARG, "NULL argument");
    const uint64_t nbpad = (h->nb + 7) / 8 * 8;
    const uint64_t need = sizeof(StoreHeader) + nbpad + h->nb * 8 + h->nchunks * sizeof(qs::ChunkMeta) + h->arena_used;
    *size = need;
    if (!buf) return QS_OK;
    if (cap < need) return fail(h, QS_ERR_ARG, "export buffer too small");
    StoreHeader hd{};
    std::memcpy(hd.magic, "QSSTORE1", 8);
    hd.n = h->n; hd.B = h->B; hd.C = h->C; hd.f64 = h->f64;
    hd.m = h->codec.m; hd.L = h->codec.L;
    hd.nb = h->nb; hd.nchunks = h->nchunks; hd.arena_bytes = h->arena_used;
    char *p = (char *)buf;
    std::memcpy(p, &hd, sizeof(hd));
    p += sizeof(hd);
    cudaStream_t s = h->stream;
    CUDA_TRY(h, cudaMemcpyAsync(p, h->mask, h->nb, cudaMemcpyDeviceToHost, s));
    p += nbpad;
    CUDA_TRY(h, cudaMemcpyAsync(p, h->block_bytes, h->nb * 8, cudaMemcpyDeviceToHost, s));
    p += h->nb * 8;
    CUDA_TRY(h, cudaMemcpyAsync(p, h->meta[h->mcur], h->nchunks * sizeof(qs::ChunkMeta), cudaMemcpyDeviceToHost, s));
    p += h->nchunks * sizeof(qs::ChunkMeta);
    if (h->arena_used) CUDA_TRY(h, cudaMemcpyAsync(p, h->arena[h->cur], h->arena_used, cudaMemcpyDefault, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    h->times[8] += 0;  // d2h time is measured by callers with their own events
    return QS_OK;
}

// True when the header of every chunk of a stored block (mask[k >> cshift])
// describes a payload of 128-byte aligned offset inside arena_bytes with a
// width of at most 32 bits.  Branch-free, split over up to eight host
// threads (a QFT n=30 store has 4 Mi headers).
static bool store_headers_valid(const uint8_t *mask, const char *meta, uint64_t nchunks, uint32_t cshift, int C,
                                uint64_t arena_bytes) {
    const uint64_t per_lane = (uint64_t)(2 << C) / 32;
    auto range_ok = [&](uint64_t k0, uint64_t k1) {
        uint64_t bad = 0;
        for (uint64_t k = k0; k < k1; ++k) {
            qs::ChunkMeta md;
            std::memcpy(&md, meta + k * sizeof(qs::ChunkMeta), sizeof(md));
            const uint64_t w = md.width;
            const uint64_t pb = ((per_lane * (w & 63) + 31) >> 5) * 128;
            const uint64_t e = (uint64_t)(w > 32) | (md.offset & 127) | (uint64_t)(md.offset > arena_bytes) |
                               (uint64_t)(pb > arena_bytes - md.offset);
            bad |= mask[k >> cshift] ? e : 0;
        }
        return bad == 0;
    };
    const unsigned nt = nchunks < (1u << 16) ? 1u : std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
    if (nt == 1) return range_ok(0, nchunks);
    std::vector<std::thread> th;
    std::vector<char> ok(nt, 1);
    const uint64_t per = (nchunks + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            const uint64_t a = std::min<uint64_t>(nchunks, t * per), b = std::min<uint64_t>(nchunks, a + per);
            ok[t] = range_ok(a, b) ? 1 : 0;
        });
    for (auto &x : th) x.join();
    for (char o : ok)
        if (!o) return false;
    return true;
}

qs_status qs_import_store(qs_state *h, const void *buf, uint64_t size) {
    if (!h || !buf) return fail(h, QS_ERR_ARG, "NULL argument");
    if (size < sizeof(StoreHeader)) return fail(h, QS_ERR_CORRUPT, "store shorter than its header");
    StoreHeader hd;
    std::memcpy(&hd, buf, sizeof(hd));
    if (std::memcmp(hd.magic, "QSSTORE1", 8) != 0 || hd.n != h->n || hd.B != h->B || hd.C != h->C ||
        hd.f64 != (uint32_t)h->f64 || hd.m != h->codec.m || hd.L != h->codec.L || hd.nb != h->nb ||
        hd.nchunks != h->nchunks)
        return fail(h, QS_ERR_CORRUPT, "store header does not match this state's geometry or codec");
    const uint64_t nbpad = (h->nb + 7) / 8 * 8;
    const uint64_t need = sizeof(StoreHeader) + nbpad + h->nb * 8 + h->nchunks * sizeof(qs::ChunkMeta) + hd.arena_bytes;
    if (size != need) return fail(h, QS_ERR_CORRUPT, "store length does not match its header");
    if (hd.arena_bytes > h->capacity) return fail(h, QS_ERR_CAPACITY, "store larger than the arena");
    const char *p = (const char *)buf + sizeof(hd);
    // every header of a stored block must describe a payload inside the
    // arena, 128-byte aligned (the decoders copy payloads with 16-byte
    // asynchronous copies); headers of unstored blocks are never read
    if (!store_headers_valid((const uint8_t *)p, p + nbpad + h->nb * 8, h->nchunks, h->B - h->C, (int)h->C,
                             hd.arena_bytes))
        return fail(h, QS_ERR_CORRUPT, "chunk header outside the stored arena");
    cudaStream_t s = h->stream;
    CUDA_TRY(h, cudaMemcpyAsync(h->mask, p, h->nb, cudaMemcpyHostToDevice, s));
    p += nbpad;
    CUDA_TRY(h, cudaMemcpyAsync(h->block_bytes, p, h->nb * 8, cudaMemcpyHostToDevice, s));
    std::vector<uint64_t> bb(h->nb);
    std::memcpy(bb.data(), p, h->nb * 8);
    p += h->nb * 8;
    CUDA_TRY(h, cudaMemcpyAsync(h->meta[h->mcur], p, h->nchunks * sizeof(qs::ChunkMeta), cudaMemcpyHostToDevice, s));
    p += h->nchunks * sizeof(qs::ChunkMeta);
    if (hd.arena_bytes) CUDA_TRY(h, cudaMemcpyAsync(h->arena[h->cur], p, hd.arena_bytes, cudaMemcpyDefault, s));
    // headers of unstored blocks were not validated: zero them on the device
    CUDA_TRY(h, qs::launch_zero_unstored_headers(h->meta[h->mcur], h->mask, h->nchunks, (int)(h->B - h->C), s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    h->arena_used = hd.arena_bytes;
    uint64_t total = 0;
    for (uint64_t v : bb) total += v;
    h->history.assign(1, total);
    return QS_OK;
}

qs_status qs_selftest_bounded_wait(uint32_t tries, int32_t *gave_up) {
    if (!gave_up || tries == 0) return fail(nullptr, QS_ERR_ARG, "gave_up must not be NULL and tries > 0");
    int32_t *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(d, 0xff, sizeof(int32_t));
    if (e == cudaSuccess) e = qs::launch_bounded_wait_selftest(tries, d, nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    int32_t v = -1;
    if (e == cudaSuccess) e = cudaMemcpy(&v, d, sizeof(v), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(nullptr, QS_ERR_CUDA, std::string("bounded-wait self-test: ") + cudaGetErrorString(e));
    }
    *gave_up = v;
    return QS_OK;
}

qs_status qs_set_zero_vector(qs_state *h) {
    if (!h) return fail(nullptr, QS_ERR_ARG, "NULL handle");
    cudaStream_t s = h->stream;
    CUDA_TRY(h, cudaMemsetAsync(h->mask, 0, h->nb, s));
    CUDA_TRY(h, cudaMemsetAsync(h->block_bytes, 0, h->nb * sizeof(unsigned long long), s));
    CUDA_TRY(h, cudaMemsetAsync(h->meta[h->mcur], 0, h->nchunks * sizeof(qs::ChunkMeta), s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    h->arena_used = 0;
    h->history.assign(1, 0);
    return QS_OK;
}

// ---- exchange of half a store across the rank boundary
// Packed layout (device memory): this 128-byte header, the half's chunk
// headers (16 bytes each), one stored flag per chunk (padded to 128 bytes),
// then the payloads (128-byte aligned, offsets in the packed headers are
// relative to the payload start).
struct HalfHeader {
    char magic[8];
    uint32_t n, B, C, f64;
    int32_t m, L;
    uint32_t qubit, value;
    uint64_t nhalf, payload_bytes;
    uint8_t pad[72];
};
static_assert(sizeof(HalfHeader) == 128, "half header is 128 bytes");

static uint64_t half_layout(uint64_t nhalf, uint64_t payload, uint64_t *meta_off, uint64_t *flags_off,
                            uint64_t *payload_off) {
    *meta_off = sizeof(HalfHeader);
    *flags_off = *meta_off + nhalf * sizeof(qs::ChunkMeta);
    *payload_off = *flags_off + (nhalf + 127) / 128 * 128;
    return *payload_off + payload;
}

static qs_status half_args(qs_state *h, uint32_t qubit, uint32_t value, qs::HalfChunks *a) {
    if (qubit < h->C || qubit >= h->n) return fail(h, QS_ERR_ARG, "exchanged qubit must lie in [chunk bits, n)");
    if (value > 1) return fail(h, QS_ERR_ARG, "half value must be 0 or 1");
    if (h->host_store) return fail(h, QS_ERR_ARG, "the exchange needs HBM arenas");
    a->bit = (int32_t)(qubit - h->C);
    a->value = value;
    a->cshift = (int32_t)(h->B - h->C);
    a->C = (int32_t)h->C;
    a->nhalf = h->nchunks / 2;
    return QS_OK;
}

}  // extern "C"

// A device allocation freed when it goes out of scope.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

extern "C" {

qs_status qs_export_half(qs_state *h, uint32_t qubit, uint32_t value, void *dev_buf, uint64_t cap, uint64_t *size) {
    if (!h || !size) return fail(h, QS_ERR_ARG, "NULL argument");
    qs::HalfChunks a{};
    qs_status st = half_args(h, qubit, value, &a);
    if (st != QS_OK) return st;
    cudaStream_t s = h->stream;
    DevBuf<uint64_t> sizes, scratch;
    DevBuf<uint8_t> flags;
    CUDA_TRY(h, cudaMalloc(&sizes.p, std::max<uint64_t>(1, a.nhalf) * 8));
    CUDA_TRY(h, cudaMalloc(&flags.p, std::max<uint64_t>(1, a.nhalf)));
    CUDA_TRY(h, cudaMalloc(&scratch.p, (qs::half_scan_scratch_words(a.nhalf) + 1) * 8));
    uint64_t *total_dev = scratch.p + qs::half_scan_scratch_words(a.nhalf);
    CUDA_TRY(h, qs::launch_half_sizes(a, h->meta[h->mcur], h->mask, sizes.p, flags.p, s));
    CUDA_TRY(h, qs::launch_half_scan(sizes.p, a.nhalf, scratch.p, total_dev, s));
    uint64_t payload = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&payload, total_dev, 8, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    uint64_t mo, fo, po;
    *size = half_layout(a.nhalf, payload, &mo, &fo, &po);
    if (!dev_buf) return QS_OK;
    if (cap < *size) return fail(h, QS_ERR_ARG, "export buffer too small");
    if ((reinterpret_cast<uintptr_t>(dev_buf) & 127) != 0) return fail(h, QS_ERR_ARG, "export buffer must be 128-byte aligned");
    HalfHeader hd{};
    std::memcpy(hd.magic, "QSHALF01", 8);
    hd.n = h->n; hd.B = h->B; hd.C = h->C; hd.f64 = h->f64;
    hd.m = h->codec.m; hd.L = h->codec.L;
    hd.qubit = qubit; hd.value = value;
    hd.nhalf = a.nhalf; hd.payload_bytes = payload;
    char *b = (char *)dev_buf;
    CUDA_TRY(h, cudaMemcpyAsync(b, &hd, sizeof(hd), cudaMemcpyHostToDevice, s));
    if (a.nhalf) CUDA_TRY(h, cudaMemcpyAsync(b + fo, flags.p, a.nhalf, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(h, qs::launch_half_pack(a, h->meta[h->mcur], h->arena[h->cur], flags.p, sizes.p,
                                     reinterpret_cast<qs::ChunkMeta *>(b + mo), reinterpret_cast<uint32_t *>(b + po),
                                     false, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    return QS_OK;
}

qs_status qs_import_half(qs_state *h, uint32_t qubit, uint32_t value, const void *dev_buf, uint64_t size) {
    if (!h || !dev_buf) return fail(h, QS_ERR_ARG, "NULL argument");
    qs::HalfChunks a{};
    qs_status st = half_args(h, qubit, value, &a);
    if (st != QS_OK) return st;
    if (size < sizeof(HalfHeader)) return fail(h, QS_ERR_CORRUPT, "exchange buffer shorter than its header");
    if ((reinterpret_cast<uintptr_t>(dev_buf) & 127) != 0) return fail(h, QS_ERR_ARG, "exchange buffer must be 128-byte aligned");
    cudaStream_t s = h->stream;
    HalfHeader hd{};
    CUDA_TRY(h, cudaMemcpyAsync(&hd, dev_buf, sizeof(hd), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    if (std::memcmp(hd.magic, "QSHALF01", 8) != 0 || hd.n != h->n || hd.B != h->B || hd.C != h->C ||
        hd.f64 != (uint32_t)h->f64 || hd.m != h->codec.m || hd.L != h->codec.L || hd.qubit != qubit ||
        hd.nhalf != a.nhalf || (hd.payload_bytes & 127) != 0)
        return fail(h, QS_ERR_CORRUPT, "exchange buffer does not match this state's geometry, codec or qubit");
    uint64_t mo, fo, po;
    if (half_layout(a.nhalf, hd.payload_bytes, &mo, &fo, &po) != size)
        return fail(h, QS_ERR_CORRUPT, "exchange buffer length does not match its header");
    const char *b = (const char *)dev_buf;
    const auto *in_meta = reinterpret_cast<const qs::ChunkMeta *>(b + mo);
    const auto *in_flags = reinterpret_cast<const uint8_t *>(b + fo);
    // every received header of a stored chunk must point inside the received payload
    CUDA_TRY(h, qs::launch_half_check(a, in_meta, in_flags, hd.payload_bytes, h->error_dev, s));
    int32_t bad = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&bad, h->error_dev, sizeof(bad), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    CUDA_TRY(h, cudaMemsetAsync(h->error_dev, 0, sizeof(int32_t), s));
    if (bad) return fail(h, QS_ERR_CORRUPT, "received chunk header outside the received payload");
    // The new store goes to the other arena: first the kept half (bit !=
    // value) compacted, then the received payloads; the replaced half's
    // payloads are left behind with the old arena.
    qs::HalfChunks kept = a;
    kept.value = value ^ 1u;
    DevBuf<uint64_t> sizes, scratch;
    DevBuf<uint8_t> flags;
    CUDA_TRY(h, cudaMalloc(&sizes.p, std::max<uint64_t>(1, a.nhalf) * 8));
    CUDA_TRY(h, cudaMalloc(&flags.p, std::max<uint64_t>(1, a.nhalf)));
    CUDA_TRY(h, cudaMalloc(&scratch.p, (qs::half_scan_scratch_words(a.nhalf) + 1) * 8));
    uint64_t *total_dev = scratch.p + qs::half_scan_scratch_words(a.nhalf);
    CUDA_TRY(h, qs::launch_half_sizes(kept, h->meta[h->mcur], h->mask, sizes.p, flags.p, s));
    CUDA_TRY(h, qs::launch_half_scan(sizes.p, a.nhalf, scratch.p, total_dev, s));
    uint64_t kept_bytes = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&kept_bytes, total_dev, 8, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    if (kept_bytes + hd.payload_bytes > h->capacity)
        return fail(h, QS_ERR_CAPACITY, "the store after the exchange does not fit the arena; set QOMPSIM_ARENA_BYTES larger");
    const int nc = h->cur ^ 1, nm = h->mcur ^ 1;
    CUDA_TRY(h, qs::launch_half_pack(kept, h->meta[h->mcur], h->arena[h->cur], flags.p, sizes.p, h->meta[nm],
                                     h->arena[nc], true, s));
    if (hd.payload_bytes)
        CUDA_TRY(h, cudaMemcpyAsync(reinterpret_cast<char *>(h->arena[nc]) + kept_bytes, b + po, hd.payload_bytes,
                                    cudaMemcpyDeviceToDevice, s));
    // received chunks: the kept half's blocks keep their stored flags (a
    // chunk-level qubit) and gain the received ones
    CUDA_TRY(h, qs::launch_half_unpack(a, in_meta, in_flags, kept_bytes, h->meta[nm], h->mask, s));
    CUDA_TRY(h, qs::launch_block_bytes(h->meta[nm], h->mask, h->nb, (int)(h->B - h->C), (int)h->C,
                                       h->block_bytes, s));
    DevBuf<unsigned long long> tot;
    CUDA_TRY(h, cudaMalloc(&tot.p, sizeof(unsigned long long)));
    CUDA_TRY(h, cudaMemsetAsync(tot.p, 0, sizeof(unsigned long long), s));
    CUDA_TRY(h, qs::launch_sum_mask_bytes(h->mask, h->block_bytes, h->nb, tot.p, s));
    unsigned long long total = 0;
    CUDA_TRY(h, cudaMemcpyAsync(&total, tot.p, sizeof(total), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(h, cudaStreamSynchronize(s));
    h->cur = nc;
    h->mcur = nm;
    h->arena_used = kept_bytes + hd.payload_bytes;
    h->history.push_back(total);
    return QS_OK;
}

}  // extern "C"

// =====================================================================
// dense state
// =====================================================================
struct qs_dense {
    uint32_t n = 0;
    bool f64 = true;
    void *state = nullptr;
    cudaStream_t stream = nullptr;
    std::string err = "no error";
    qs::KGate *kg = nullptr;
    size_t kg_cap = 0;
    qs::Sweep *sw = nullptr;
    size_t sw_cap = 0;
    qs::ROp *ops = nullptr;
    size_t ops_cap = 0;
    void *pool = nullptr;
    size_t pool_cap = 0;  // bytes
    double *dscratch = nullptr;
    ~qs_dense() {
        if (state) cudaFree(state);
        if (kg) cudaFree(kg);
        if (sw) cudaFree(sw);
        if (ops) cudaFree(ops);
        if (pool) cudaFree(pool);
        if (dscratch) cudaFree(dscratch);
    }
    uint64_t dim() const { return uint64_t(1) << n; }
    size_t amp_bytes() const { return f64 ? 16 : 8; }
};

static qs_status dfail(qs_dense *h, qs_status s, const std::string &m) {
    if (h) h->err = m;
    else g_last_error = m;
    return s;
}

static qs_status dense_upload_gates(qs_dense *h, const std::vector<qs::KGate> &kg) {
    if (kg.size() > h->kg_cap) {
        if (h->kg) cudaFree(h->kg);
        h->kg = nullptr;
        h->kg_cap = 0;
        CUDA_TRY(h, cudaMalloc(&h->kg, kg.size() * sizeof(qs::KGate)));
        h->kg_cap = kg.size();
    }
    if (!kg.empty())
        CUDA_TRY(h, cudaMemcpyAsync(h->kg, kg.data(), kg.size() * sizeof(qs::KGate), cudaMemcpyHostToDevice, h->stream));
    return QS_OK;
}

extern "C" {

const char *qs_dense_last_error(const qs_dense *h) { return h ? h->err.c_str() : g_last_error.c_str(); }

qs_status qs_dense_create(qs_dense **out, uint32_t n, qs_dtype dtype) {
    if (!out) return dfail(nullptr, QS_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n < 1 || n > 36) return dfail(nullptr, QS_ERR_ARG, "need 1 <= n <= 36");
    if (dtype != QS_COMPLEX128 && dtype != QS_COMPLEX64) return dfail(nullptr, QS_ERR_ARG, "unknown dtype");
    auto *h = new (std::nothrow) qs_dense();
    if (!h) return dfail(nullptr, QS_ERR_NOMEM, "host allocation failed");
    h->n = n;
    h->f64 = dtype == QS_COMPLEX128;
    cudaError_t e = cudaMalloc(&h->state, h->dim() * h->amp_bytes());
    if (e == cudaSuccess) e = cudaMalloc(&h->dscratch, 4 * sizeof(double));
    if (e != cudaSuccess) {
        std::string m = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        delete h;
        return dfail(nullptr, e == cudaErrorMemoryAllocation ? QS_ERR_CAPACITY : QS_ERR_CUDA, m);
    }
    qs_status s = qs_dense_set_basis_state(h, 0);
    if (s != QS_OK) {
        std::string m = h->err;
        delete h;
        return dfail(nullptr, s, m);
    }
    *out = h;
    return QS_OK;
}

qs_status qs_dense_destroy(qs_dense *h) {
    delete h;
    return QS_OK;
}

qs_status qs_dense_set_stream(qs_dense *h, void *stream) {
    if (!h) return dfail(nullptr, QS_ERR_ARG, "NULL handle");
    h->stream = (cudaStream_t)stream;
    return QS_OK;
}

qs_status qs_dense_set_basis_state(qs_dense *h, uint64_t basis) {
    if (!h) return dfail(nullptr, QS_ERR_ARG, "NULL handle");
    if (basis >> h->n) return dfail(h, QS_ERR_ARG, "basis index out of range");
    CUDA_TRY(h, cudaMemsetAsync(h->state, 0, h->dim() * h->amp_bytes(), h->stream));
    if (h->f64) {
        const double one[2] = {1.0, 0.0};
        CUDA_TRY(h, cudaMemcpyAsync((char *)h->state + basis * 16, one, 16, cudaMemcpyHostToDevice, h->stream));
    } else {
        const float one[2] = {1.0f, 0.0f};
        CUDA_TRY(h, cudaMemcpyAsync((char *)h->state + basis * 8, one, 8, cudaMemcpyHostToDevice, h->stream));
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

static qs_status dense_canon(qs_dense *h, const qs_gate *gates, size_t count, std::vector<CGate> *cg) {
    cg->resize(count);
    for (size_t i = 0; i < count; ++i) {
        std::string e;
        if (!canonicalize(gates[i], false, h->n, &(*cg)[i], &e))
            return dfail(h, e.find("index") != std::string::npos ? QS_ERR_ARG : QS_ERR_UNSUPPORTED_GATE,
                         "gate " + std::to_string(i) + ": " + e);
    }
    return QS_OK;
}

qs_status qs_dense_apply_gates(qs_dense *h, const qs_gate *gates, size_t count) {
    if (!h) return dfail(nullptr, QS_ERR_ARG, "NULL handle");
    if (count && !gates) return dfail(h, QS_ERR_ARG, "gates is NULL");
    if (!count) return QS_OK;
    std::vector<CGate> cg;
    qs_status s = dense_canon(h, gates, count, &cg);
    if (s != QS_OK) return s;
    const int C = (int)std::min<uint32_t>(h->n, (uint32_t)env_int("QOMPSIM_DENSE_CHUNK_LOG2", 5));
    const int tl = env_int("QOMPSIM_DENSE_TILE_LOG2", h->f64 ? 12 : 13);
    const int tile_log2 = std::min<int>((int)h->n, std::min<int>(tl, C + qs::kMaxTileQubits));
    const int jmax = tile_log2 - C;
    const int RB = qs::kRegBits;
    if ((int)h->n < RB) return qs_dense_apply_gates_pergate(h, gates, count);
    std::vector<uint32_t> ids(count);
    for (size_t i = 0; i < count; ++i) ids[i] = (uint32_t)i;
    auto pl = env_int("QOMPSIM_DAG_PLAN", 1) ? plan_passes_dag(ids, cg, C, jmax, std::min(jmax, 3), C, (int)h->n)
                                             : plan_passes(ids, cg, C, jmax, std::min(jmax, 3), C, (int)h->n);
    std::vector<qs::KGate> kg;
    std::vector<qs::Sweep> sw;
    std::vector<qs::ROp> ops;
    std::vector<cplx> pool;
    std::vector<std::pair<size_t, size_t>> sweep_ranges;
    std::vector<size_t> op_offsets;
    std::vector<std::vector<int>> outers;
    for (auto &p : pl) {
        // a tile must hold at least the RB register bits
        std::set<int> t(p.tile.begin(), p.tile.end());
        for (int q = C; q < (int)h->n && C + (int)t.size() < RB; ++q) t.insert(q);
        p.tile.assign(t.begin(), t.end());
        const size_t g0 = kg.size();
        for (uint32_t gi : p.gates) kg.push_back(to_kgate(cg[gi], p.tile, C));
        auto swp = plan_sweeps(kg, g0, kg.size(), C + (int)p.tile.size(), RB);
        const size_t op0 = ops.size();
        std::vector<RawOp> raw;
        std::vector<cplx> rpool;
        build_ops(kg, g0, swp, RB, &raw, &rpool);
        std::vector<qs::Sweep> merged;
        merge_diagonal_ops(swp, 0, &raw, &rpool, &merged);
        swp.swap(merged);
        std::vector<int> outer;
        if (!finalize_ops(raw, rpool, C + (int)p.tile.size(), &outer, &ops, &pool))
            return dfail(h, QS_ERR_ARG, "a pass needs more outer selector qubits than the planner allows");
        fuse_half_chains(&ops, op0, swp);
        outers.push_back(outer);
        op_offsets.push_back(op0);
        sweep_ranges.push_back({sw.size(), swp.size()});
        sw.insert(sw.end(), swp.begin(), swp.end());
    }
    if (ops.size() > h->ops_cap) {
        if (h->ops) cudaFree(h->ops);
        h->ops = nullptr;
        h->ops_cap = 0;
        CUDA_TRY(h, cudaMalloc(&h->ops, ops.size() * sizeof(qs::ROp)));
        h->ops_cap = ops.size();
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->ops, ops.data(), ops.size() * sizeof(qs::ROp), cudaMemcpyHostToDevice, h->stream));
    {
        const size_t bytes = pool.size() * 2 * (h->f64 ? sizeof(double) : sizeof(float));
        if (bytes > h->pool_cap) {
            if (h->pool) cudaFree(h->pool);
            h->pool = nullptr;
            h->pool_cap = 0;
            CUDA_TRY(h, cudaMalloc(&h->pool, bytes));
            h->pool_cap = bytes;
        }
        if (h->f64) {
            auto pv = pool_as<double>(pool);
            CUDA_TRY(h, cudaMemcpy(h->pool, pv.data(), bytes, cudaMemcpyHostToDevice));
        } else {
            auto pv = pool_as<float>(pool);
            CUDA_TRY(h, cudaMemcpy(h->pool, pv.data(), bytes, cudaMemcpyHostToDevice));
        }
    }
    if (sw.size() > h->sw_cap) {
        if (h->sw) cudaFree(h->sw);
        h->sw = nullptr;
        h->sw_cap = 0;
        CUDA_TRY(h, cudaMalloc(&h->sw, sw.size() * sizeof(qs::Sweep)));
        h->sw_cap = sw.size();
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->sw, sw.data(), sw.size() * sizeof(qs::Sweep), cudaMemcpyHostToDevice, h->stream));
    size_t off = 0;
    for (size_t pi = 0; pi < pl.size(); ++pi) {
        auto &p = pl[pi];
        qs::DensePassArgs a{};
        a.n = (int)h->n;
        a.C = C;
        a.j = (int)p.tile.size();
        for (int k = 0; k < a.j; ++k) a.tq[k] = p.tile[k] - C;
        a.n_tiles = uint64_t(1) << (h->n - C - a.j);
        a.ops = h->ops + op_offsets[pi];
        a.pool = h->pool;
        a.sweeps = h->sw + sweep_ranges[pi].first;
        a.nsweeps = (int)sweep_ranges[pi].second;
        a.rb = RB;
        a.nouter = (int)outers[pi].size();
        for (size_t k = 0; k < outers[pi].size(); ++k) a.outer_q[k] = (int8_t)outers[pi][k];
        a.state = h->state;
        off += p.gates.size();
        CUDA_TRY(h, qs::launch_dense_pass(h->f64, a, tile_log2, h->stream));
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_dense_apply_gates_pergate(qs_dense *h, const qs_gate *gates, size_t count) {
    if (!h) return dfail(nullptr, QS_ERR_ARG, "NULL handle");
    if (count && !gates) return dfail(h, QS_ERR_ARG, "gates is NULL");
    if (!count) return QS_OK;
    std::vector<CGate> cg;
    qs_status s = dense_canon(h, gates, count, &cg);
    if (s != QS_OK) return s;
    if (h->n < 2) {
        for (auto &g : cg)
            if (g.nq == 2) return dfail(h, QS_ERR_ARG, "two-qubit gate on a one-qubit state");
    }
    std::vector<qs::KGate> kg;
    for (auto &g : cg) kg.push_back(to_kgate(g, {}, 64));
    s = dense_upload_gates(h, kg);
    if (s != QS_OK) return s;
    for (size_t i = 0; i < kg.size(); ++i) CUDA_TRY(h, qs::launch_pergate(h->f64, h->state, (int)h->n, h->kg + i, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_dense_get_amplitudes(qs_dense *h, uint64_t first, uint64_t count, double *out) {
    if (!h || (count && !out)) return dfail(h, QS_ERR_ARG, "NULL argument");
    if (first > h->dim() || count > h->dim() - first) return dfail(h, QS_ERR_ARG, "amplitude range outside the state");
    if (!count) return QS_OK;
    if (h->f64) {
        CUDA_TRY(h, cudaMemcpyAsync(out, static_cast<const double *>(h->state) + 2 * first, count * 16,
                                    cudaMemcpyDefault, h->stream));
    } else {
        double *tmp = nullptr;
        CUDA_TRY(h, cudaMalloc(&tmp, count * 16));
        cudaError_t e = qs::launch_dense_to_c128(false, static_cast<const float *>(h->state) + 2 * first, count, tmp,
                                                 h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, count * 16, cudaMemcpyDefault, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            return dfail(h, QS_ERR_CUDA, std::string("get_amplitudes: ") + cudaGetErrorString(e));
        }
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_dense_get_vector(qs_dense *h, double *out) {
    if (!h || !out) return dfail(h, QS_ERR_ARG, "NULL argument");
    if (h->f64) {
        CUDA_TRY(h, cudaMemcpyAsync(out, h->state, h->dim() * 16, cudaMemcpyDeviceToHost, h->stream));
    } else {
        double *tmp = nullptr;
        CUDA_TRY(h, cudaMalloc(&tmp, h->dim() * 16));
        cudaError_t e = qs::launch_dense_to_c128(false, h->state, h->dim(), tmp, h->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, h->dim() * 16, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) return dfail(h, QS_ERR_CUDA, std::string("get_vector: ") + cudaGetErrorString(e));
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_dense_set_vector(qs_dense *h, const double *in) {
    if (!h || !in) return dfail(h, QS_ERR_ARG, "NULL argument");
    if (h->f64) {
        CUDA_TRY(h, cudaMemcpyAsync(h->state, in, h->dim() * 16, cudaMemcpyHostToDevice, h->stream));
    } else {
        double *tmp = nullptr;
        CUDA_TRY(h, cudaMalloc(&tmp, h->dim() * 16));
        cudaError_t e = cudaMemcpyAsync(tmp, in, h->dim() * 16, cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = qs::launch_c128_to_dense(false, tmp, h->dim(), h->state, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) return dfail(h, QS_ERR_CUDA, std::string("set_vector: ") + cudaGetErrorString(e));
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_dense_norm_squared(qs_dense *h, double *out) {
    if (!h || !out) return dfail(h, QS_ERR_ARG, "NULL argument");
    CUDA_TRY(h, cudaMemsetAsync(h->dscratch, 0, sizeof(double), h->stream));
    CUDA_TRY(h, qs::launch_dense_norm(h->f64, h->state, h->dim(), h->dscratch, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(out, h->dscratch, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return QS_OK;
}

qs_status qs_dense_device_ptr(qs_dense *h, void **out) {
    if (!h || !out) return dfail(h, QS_ERR_ARG, "NULL argument");
    *out = h->state;
    return QS_OK;
}

qs_status qs_dense_expectation_pauli(qs_dense *h, const uint64_t *x_masks, const uint64_t *z_masks, size_t nterms,
                                     double *out) {
    if (!h || (nterms && (!x_masks || !z_masks || !out))) return dfail(h, QS_ERR_ARG, "NULL argument");
    const uint64_t full = h->n >= 64 ? ~0ull : ((1ull << h->n) - 1);
    std::vector<qs::PauliTerm> pts(nterms);
    for (size_t t = 0; t < nterms; ++t) {
        if ((x_masks[t] | z_masks[t]) & ~full) return dfail(h, QS_ERR_ARG, "Pauli term acts outside the register");
        pts[t] = qs::PauliTerm{};
        pts[t].xg = x_masks[t];
        pts[t].zg = z_masks[t];
    }
    if (!nterms) return QS_OK;
    qs::PauliTerm *dt = nullptr;
    double *dout = nullptr;
    cudaError_t e = cudaMalloc(&dt, nterms * sizeof(qs::PauliTerm));
    if (e == cudaSuccess) e = cudaMalloc(&dout, 2 * nterms * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, pts.data(), nterms * sizeof(qs::PauliTerm), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dout, 0, 2 * nterms * sizeof(double), h->stream);
    for (size_t t0 = 0; t0 < nterms && e == cudaSuccess; t0 += 256) {
        const int cnt = (int)std::min<size_t>(256, nterms - t0);
        e = qs::launch_dense_expect(h->f64, h->state, (int)h->n, dt + t0, cnt, dout + 2 * t0, h->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, 2 * nterms * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (dt) cudaFree(dt);
    if (dout) cudaFree(dout);
    if (e != cudaSuccess) return dfail(h, QS_ERR_CUDA, std::string("expectation: ") + cudaGetErrorString(e));
    return QS_OK;
}

qs_status qs_dense_copy(qs_dense *dst, const qs_dense *src) {
    if (!dst || !src) return dfail(dst, QS_ERR_ARG, "NULL handle");
    if (dst->n != src->n || dst->f64 != src->f64) return dfail(dst, QS_ERR_ARG, "states differ in size or dtype");
    CUDA_TRY(dst, cudaMemcpyAsync(dst->state, src->state, dst->dim() * dst->amp_bytes(), cudaMemcpyDeviceToDevice,
                                  dst->stream));
    CUDA_TRY(dst, cudaStreamSynchronize(dst->stream));
    return QS_OK;
}

static qs_status pauli_terms(qs_dense *h, const uint64_t *x, const uint64_t *z, size_t nterms,
                             std::vector<qs::PauliTerm> *out) {
    const uint64_t full = h->n >= 64 ? ~0ull : ((1ull << h->n) - 1);
    out->resize(nterms);
    for (size_t t = 0; t < nterms; ++t) {
        if ((x[t] | z[t]) & ~full) return dfail(h, QS_ERR_ARG, "Pauli term acts outside the register");
        (*out)[t] = qs::PauliTerm{};
        (*out)[t].xg = x[t];
        (*out)[t].zg = z[t];
    }
    return QS_OK;
}

qs_status qs_dense_apply_pauli_sum(qs_dense *out, const qs_dense *in, const uint64_t *x_masks, const uint64_t *z_masks,
                                   const double *coefs, size_t nterms) {
    if (!out || !in || (nterms && (!x_masks || !z_masks || !coefs))) return dfail(out, QS_ERR_ARG, "NULL argument");
    if (out == in) return dfail(out, QS_ERR_ARG, "in and out must be different states");
    if (out->n != in->n || out->f64 != in->f64) return dfail(out, QS_ERR_ARG, "states differ in size or dtype");
    std::vector<qs::PauliTerm> pts;
    qs_status st = pauli_terms(out, x_masks, z_masks, nterms, &pts);
    if (st != QS_OK) return st;
    qs::PauliTerm *dt = nullptr;
    double *dc = nullptr;
    cudaError_t e = cudaMalloc(&dt, std::max<size_t>(1, nterms) * sizeof(qs::PauliTerm));
    if (e == cudaSuccess) e = cudaMalloc(&dc, std::max<size_t>(1, 2 * nterms) * sizeof(double));
    if (e == cudaSuccess && nterms)
        e = cudaMemcpyAsync(dt, pts.data(), nterms * sizeof(qs::PauliTerm), cudaMemcpyHostToDevice, out->stream);
    if (e == cudaSuccess && nterms)
        e = cudaMemcpyAsync(dc, coefs, 2 * nterms * sizeof(double), cudaMemcpyHostToDevice, out->stream);
    if (e == cudaSuccess)
        e = qs::launch_dense_pauli_sum(out->f64, in->state, out->state, (int)out->n, dt, dc, (int)nterms, out->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(out->stream);
    if (dt) cudaFree(dt);
    if (dc) cudaFree(dc);
    if (e != cudaSuccess) return dfail(out, QS_ERR_CUDA, std::string("apply_pauli_sum: ") + cudaGetErrorString(e));
    return QS_OK;
}

qs_status qs_dense_transition_pauli(const qs_dense *bra, qs_dense *ket, const uint64_t *x_masks,
                                    const uint64_t *z_masks, size_t nterms, double *out) {
    if (!bra || !ket || (nterms && (!x_masks || !z_masks || !out))) return dfail(ket, QS_ERR_ARG, "NULL argument");
    if (bra->n != ket->n || bra->f64 != ket->f64) return dfail(ket, QS_ERR_ARG, "states differ in size or dtype");
    std::vector<qs::PauliTerm> pts;
    qs_status st = pauli_terms(ket, x_masks, z_masks, nterms, &pts);
    if (st != QS_OK || !nterms) return st;
    qs::PauliTerm *dt = nullptr;
    double *dout = nullptr;
    cudaError_t e = cudaMalloc(&dt, nterms * sizeof(qs::PauliTerm));
    if (e == cudaSuccess) e = cudaMalloc(&dout, 2 * nterms * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, pts.data(), nterms * sizeof(qs::PauliTerm), cudaMemcpyHostToDevice, ket->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dout, 0, 2 * nterms * sizeof(double), ket->stream);
    for (size_t t0 = 0; t0 < nterms && e == cudaSuccess; t0 += 256) {
        const int cnt = (int)std::min<size_t>(256, nterms - t0);
        e = qs::launch_dense_transition(ket->f64, bra->state, ket->state, (int)ket->n, dt + t0, cnt, dout + 2 * t0,
                                        ket->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, 2 * nterms * sizeof(double), cudaMemcpyDeviceToHost, ket->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ket->stream);
    if (dt) cudaFree(dt);
    if (dout) cudaFree(dout);
    if (e != cudaSuccess) return dfail(ket, QS_ERR_CUDA, std::string("transition: ") + cudaGetErrorString(e));
    return QS_OK;
}

// Fused adjoint backward sweep over psi and lam (see qompsim.h).
qs_status qs_dense_adjoint(qs_dense *psi, qs_dense *lam, const qs_gate *gates, const int32_t *slots,
                           const uint64_t *gen_x, const uint64_t *gen_z, size_t count, double *out, uint32_t nslots) {
    if (!psi || !lam || (count && (!gates || !slots || !gen_x || !gen_z)) || (nslots && !out))
        return dfail(psi, QS_ERR_ARG, "NULL argument");
    if (psi == lam || psi->n != lam->n || psi->f64 != lam->f64)
        return dfail(psi, QS_ERR_ARG, "psi and lam must be distinct states of one size and dtype");
    if (psi->stream != lam->stream) return dfail(psi, QS_ERR_ARG, "psi and lam must share a stream");
    for (size_t i = 0; i < count; ++i)
        if (slots[i] >= (int32_t)nslots) return dfail(psi, QS_ERR_ARG, "slot index out of range");
    std::vector<CGate> cg;
    qs_status st = dense_canon(psi, gates, count, &cg);
    if (st != QS_OK) return st;
    const int n = (int)psi->n;
    const int C = std::min(n, 5);
    const int tile_log2 = std::min(n, std::min(psi->f64 ? 11 : 12, C + qs::kMaxTileQubits));
    const int jmax = tile_log2 - C;
    // generators' flip qubits must lie in the tile too: treat them as mixing
    for (size_t i = 0; i < count; ++i)
        if (slots[i] >= 0)
            for (int b = 0; b < cg[i].nq; ++b)
                if ((gen_x[i] >> cg[i].q[b]) & 1) cg[i].mix[b] = true;
    for (size_t i = 0; i < count; ++i) {
        uint64_t covered = 0;
        for (int b = 0; b < cg[i].nq; ++b) covered |= 1ull << cg[i].q[b];
        if (slots[i] >= 0 && (gen_x[i] & ~covered))
            return dfail(psi, QS_ERR_ARG, "a generator flips a qubit its gate does not act on");
    }
    std::vector<uint32_t> ids(count);
    for (size_t i = 0; i < count; ++i) ids[i] = (uint32_t)i;
    // commuting gates may change places (the argument at qs_adjoint holds here)
    auto pl = env_int("QOMPSIM_DAG_PLAN", 1) ? plan_passes_dag(ids, cg, C, jmax, std::min(jmax, 3), C, n)
                                             : plan_passes(ids, cg, C, jmax, std::min(jmax, 3), C, n);
    // every launch's gate records (at most 128 parametric gates each) are
    // built first and uploaded at once; the launches then run back to back
    // and their slot sums are read back with one copy at the end
    struct Launch {
        int j;
        int32_t tq[qs::kMaxTileQubits];
        size_t gate_off, ngates, out_off;
        std::vector<int32_t> local_to_global;
        std::vector<int> tile;
        std::vector<uint32_t> gates;
        bool fused = false;
        DualSweepPlan sweeps;
    };
    std::vector<qs::AdjGate> ag;
    std::vector<Launch> launches;
    size_t nout = 0;
    for (auto &p : pl) {
        for (size_t g0 = 0; g0 < p.gates.size();) {
            Launch L{};
            L.j = (int)p.tile.size();
            for (int k = 0; k < L.j; ++k) L.tq[k] = p.tile[k] - C;
            L.tile = p.tile;
            L.gate_off = ag.size();
            L.out_off = nout;
            size_t g1 = g0;
            for (; g1 < p.gates.size(); ++g1) {
                const uint32_t gi = p.gates[g1];
                if (slots[gi] >= 0 && L.local_to_global.size() >= 128) break;
                qs::AdjGate a{};
                a.g = to_kgate(cg[gi], p.tile, C);
                a.slot = -1;
                if (slots[gi] >= 0) {
                    a.slot = (int32_t)L.local_to_global.size();
                    L.local_to_global.push_back(slots[gi]);
                    uint32_t xt = 0, zt = 0;
                    uint64_t zo = 0;
                    for (int q = 0; q < n; ++q) {
                        int tp = q < C ? q : -1;
                        if (q >= C) {
                            auto it = std::find(p.tile.begin(), p.tile.end(), q);
                            if (it != p.tile.end()) tp = C + (int)(it - p.tile.begin());
                        }
                        if ((gen_x[gi] >> q) & 1) xt |= 1u << tp;  // flip qubits are in the tile
                        if ((gen_z[gi] >> q) & 1) {
                            if (tp >= 0) zt |= 1u << tp;
                            else zo |= 1ull << q;
                        }
                    }
                    a.gen.xt = xt;
                    a.gen.zt = zt;
                    a.gen.zo = zo;
                }
                ag.push_back(a);
                L.gates.push_back(gi);
            }
            L.ngates = ag.size() - L.gate_off;
            nout += L.local_to_global.size();
            launches.push_back(std::move(L));
            g0 = g1;
        }
    }
    // register sweeps over both tiles (the shared-memory op path stays for
    // launches the sweeps cannot express, and behind QOMPSIM_DUAL_SWEEPS=0)
    const int RB = psi->f64 ? qs::kDualRegBitsF64 : qs::kDualRegBitsF32;
    std::vector<qs::Sweep> all_sw;
    std::vector<qs::ROp> all_rops;
    std::vector<cplx> all_pool;
    if (env_int("QOMPSIM_DUAL_SWEEPS", 1))
        for (Launch &L : launches)
            L.fused = plan_dual_sweeps(cg, L.gates, slots, gen_x, gen_z, L.tile, C, RB, &all_sw, &all_rops, &all_pool,
                                       &L.sweeps);
    std::vector<double> acc(2 * (size_t)nslots, 0.0);
    double *dout = nullptr;
    qs::AdjGate *dg = nullptr;
    qs::Sweep *dsw = nullptr;
    qs::ROp *drops = nullptr;
    void *dpool = nullptr;
    const size_t pool_bytes = all_pool.size() * (psi->f64 ? 16 : 8);
    std::vector<float> pool_f;
    std::vector<double> pool_d;
    if (psi->f64) pool_d = pool_as<double>(all_pool);
    else pool_f = pool_as<float>(all_pool);
    cudaError_t e = cudaMalloc(&dg, std::max<size_t>(1, ag.size()) * sizeof(qs::AdjGate));
    if (e == cudaSuccess) e = cudaMalloc(&dout, std::max<size_t>(1, 2 * nout) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dsw, std::max<size_t>(1, all_sw.size()) * sizeof(qs::Sweep));
    if (e == cudaSuccess) e = cudaMalloc(&drops, std::max<size_t>(1, all_rops.size()) * sizeof(qs::ROp));
    if (e == cudaSuccess) e = cudaMalloc(&dpool, std::max<size_t>(16, pool_bytes));
    if (e == cudaSuccess && !ag.empty())
        e = cudaMemcpyAsync(dg, ag.data(), ag.size() * sizeof(qs::AdjGate), cudaMemcpyHostToDevice, psi->stream);
    if (e == cudaSuccess && !all_sw.empty())
        e = cudaMemcpyAsync(dsw, all_sw.data(), all_sw.size() * sizeof(qs::Sweep), cudaMemcpyHostToDevice,
                            psi->stream);
    if (e == cudaSuccess && !all_rops.empty())
        e = cudaMemcpyAsync(drops, all_rops.data(), all_rops.size() * sizeof(qs::ROp), cudaMemcpyHostToDevice,
                            psi->stream);
    if (e == cudaSuccess && pool_bytes)
        e = cudaMemcpyAsync(dpool, psi->f64 ? (const void *)pool_d.data() : (const void *)pool_f.data(), pool_bytes,
                            cudaMemcpyHostToDevice, psi->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dout, 0, std::max<size_t>(1, 2 * nout) * sizeof(double), psi->stream);
    for (const Launch &L : launches) {
        if (e != cudaSuccess) break;
        qs::AdjPassArgs a{};
        if (L.fused) {
            a.sweeps = dsw + L.sweeps.sw_off;
            a.nsweeps = (int32_t)L.sweeps.nsw;
            a.rb = RB;
            a.rops = drops + L.sweeps.rop_off;
            a.pool = dpool;
            a.nouter = (int32_t)L.sweeps.outer.size();
            for (int i = 0; i < a.nouter; ++i) a.outer_q[i] = (int8_t)L.sweeps.outer[i];
        }
        a.n = n;
        a.C = C;
        a.j = L.j;
        for (int k = 0; k < L.j; ++k) a.tq[k] = L.tq[k];
        a.n_tiles = uint64_t(1) << (n - C - L.j);
        a.gates = dg + L.gate_off;
        a.ngates = (int)L.ngates;
        a.psi = psi->state;
        a.lam = lam->state;
        a.out = dout + 2 * L.out_off;
        a.nslots = (int)L.local_to_global.size();
        e = qs::launch_adjoint_pass(psi->f64, a, psi->stream);
    }
    std::vector<double> h(2 * nout);
    if (e == cudaSuccess && nout)
        e = cudaMemcpyAsync(h.data(), dout, 2 * nout * sizeof(double), cudaMemcpyDeviceToHost, psi->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(psi->stream);
    if (e == cudaSuccess)
        for (const Launch &L : launches)
            for (size_t k = 0; k < L.local_to_global.size(); ++k) {
                acc[2 * L.local_to_global[k]] += h[2 * (L.out_off + k)];
                acc[2 * L.local_to_global[k] + 1] += h[2 * (L.out_off + k) + 1];
            }
    if (dg) cudaFree(dg);
    if (dout) cudaFree(dout);
    if (dsw) cudaFree(dsw);
    if (drops) cudaFree(drops);
    if (dpool) cudaFree(dpool);
    if (e != cudaSuccess) return dfail(psi, QS_ERR_CUDA, std::string("adjoint: ") + cudaGetErrorString(e));
    for (size_t i = 0; i < acc.size(); ++i) out[i] = acc[i];
    return QS_OK;
}

// Device codec round trip used by the CPU/GPU bit-identity tests.
qs_status qs_codec_test(qs_dtype dtype, double eps_rel, double eps_abs, uint32_t chunk_log2, const void *vals,
                        uint64_t nchunks, uint32_t *words, int32_t *bases, uint32_t *widths, void *decoded) {
    qs::CodecParams p;
    const bool f64 = dtype == QS_COMPLEX128;
    if (!qs::codec_params(f64, eps_rel, eps_abs, &p)) return dfail(nullptr, QS_ERR_ARG, "bad error bounds");
    if (chunk_log2 < (uint32_t)qs::kMinChunkLog2 || chunk_log2 > (uint32_t)qs::kMaxChunkLog2 || !vals || !words ||
        !bases || !widths || !decoded)
        return dfail(nullptr, QS_ERR_ARG, "bad argument");
    const uint64_t ncomp = (uint64_t(2) << chunk_log2) * nchunks;
    const size_t rsz = f64 ? 8 : 4;
    const uint64_t max_words = (uint64_t(2) << chunk_log2) * nchunks;  // width 32 -> one word per component
    void *dv = nullptr, *dd = nullptr;
    uint32_t *dw = nullptr;
    int32_t *db = nullptr;
    uint32_t *dwi = nullptr;
    cudaError_t e = cudaMalloc(&dv, ncomp * rsz);
    if (e == cudaSuccess) e = cudaMalloc(&dd, ncomp * rsz);
    if (e == cudaSuccess) e = cudaMalloc(&dw, max_words * 4);
    if (e == cudaSuccess) e = cudaMalloc(&db, nchunks * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dwi, nchunks * 4);
    if (e == cudaSuccess) e = cudaMemset(dw, 0, max_words * 4);
    if (e == cudaSuccess) e = cudaMemcpy(dv, vals, ncomp * rsz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = qs::launch_codec_test(f64, dv, (int)chunk_log2, p, nchunks, dw, db, dwi, dd, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(words, dw, max_words * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(bases, db, nchunks * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(widths, dwi, nchunks * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(decoded, dd, ncomp * rsz, cudaMemcpyDeviceToHost);
    cudaFree(dv);
    cudaFree(dd);
    cudaFree(dw);
    cudaFree(db);
    cudaFree(dwi);
    if (e != cudaSuccess) return dfail(nullptr, QS_ERR_CUDA, std::string("codec test: ") + cudaGetErrorString(e));
    return QS_OK;
}

// Allocation-free codec round trip (see qompsim.h): device pointers in and
// out, scratch in a file-scope device array, no cudaMalloc / cudaFree.
qs_status qs_codec_roundtrip_noalloc(qs_dtype dtype, double eps_rel, double eps_abs, uint32_t chunk_log2,
                                     const void *d_vals, uint64_t nchunks, int32_t *d_bases, uint32_t *d_widths,
                                     void *d_decoded, void *stream) {
    qs::CodecParams p;
    if (dtype != QS_COMPLEX128 && dtype != QS_COMPLEX64) return dfail(nullptr, QS_ERR_ARG, "unknown dtype");
    const bool f64 = dtype == QS_COMPLEX128;
    if (!qs::codec_params(f64, eps_rel, eps_abs, &p))
        return dfail(nullptr, QS_ERR_ARG, "eps_rel must lie in [2^-24, 1)");
    if (chunk_log2 < (uint32_t)qs::kMinChunkLog2 || chunk_log2 > (uint32_t)qs::kMaxChunkLog2)
        return dfail(nullptr, QS_ERR_ARG, "chunk_log2 must lie in [4, 8]");
    if (nchunks == 0) return QS_OK;
    if (!d_vals || !d_bases || !d_widths || !d_decoded) return dfail(nullptr, QS_ERR_ARG, "NULL device pointer");
    const uint64_t words_per_chunk = uint64_t(2) << chunk_log2;
    const uint64_t cap = qs::noalloc_scratch_words();
    if (nchunks > cap / words_per_chunk)
        return dfail(nullptr, QS_ERR_ARG,
                     "qs_codec_roundtrip_noalloc: " + std::to_string(nchunks) + " chunks of 2^" +
                         std::to_string(chunk_log2) + " amplitudes exceed its fixed scratch of " +
                         std::to_string(cap * 4) + " bytes (at most " + std::to_string(cap / words_per_chunk) +
                         " chunks per call)");
    cudaError_t e = qs::launch_codec_roundtrip_noalloc(f64, d_vals, (int)chunk_log2, p, nchunks, d_bases, d_widths,
                                                       d_decoded, (cudaStream_t)stream);
    if (e != cudaSuccess)
        return dfail(nullptr, QS_ERR_CUDA, std::string("qs_codec_roundtrip_noalloc: ") + cudaGetErrorString(e));
    return QS_OK;
}

}  // extern "C"
