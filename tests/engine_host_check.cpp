// CPU check of host logic of the engine that the device tests only reach
// indirectly.  Compiled together with engine.cpp (included below) by
// tests/test_engine_host.py; nothing here touches a GPU: the planner's host
// step (plan_device_passes) uploads nothing, and the store-header check is
// host code.
//
//   engine_host_check headers
//       store_headers_valid: valid stores pass; a misaligned offset, a width
//       above 32, a payload past the arena fail; unstored blocks are ignored
//   engine_host_check plan <gates file> <n> <B> <I> <f64>
//       prints one line per device pass: kind (0 tile, 1 chunk headers), tile
//       qubits j, code-domain flag (every op an X / SWAP move), and the
//       largest tile j of the precision
//   engine_host_check tail <gates file> <n> <B> <I> <f64>
//       per start stage: passes of the per-stage plan from there, passes of
//       the merged tail, and the tail pass that ends each stage
//   engine_host_check selruns
//       encode_selector_runs on random selector sets: where the selectors
//       form at most two runs of consecutive bits, the variant computed from
//       the runs picks, for every selector word, the matrix entries that the
//       per-bit variant of the original selectors picked; other sets are
//       left as they were
//   engine_host_check dagplan
//       plan_passes_dag and plan_passes on random gate lists: every gate is
//       placed once; a pass's tile holds every qubit >= C on which one of its
//       gates mixes amplitudes and at most jmax of them (padded to jmin);
//       its other qubits >= C fit the outer selectors; and the passes' gates
//       in order keep every two gates that do not commute (they share a qubit
//       on which one of them mixes) in their original order
//   engine_host_check chunkperm
//       stage_relabel on random gate lists: SWAP and X gates on qubits >= C
//       fold into a chunk permutation and the other gates are relabelled
//       through it; the relabelled gates followed by the permutation's chunk
//       moves give the original list's state on a dense vector
//   engine_host_check opcompile
//       the fused path's op compiler (planner, sweeps, register ops,
//       diagonal merging, selector variants, chain fusion) on random
//       circuits: its ops, interpreted over every tile of a dense vector by a
//       host restatement of the tile pass, give the gates applied one by one
//   engine_host_check dualcompile
//       the two-store (adjoint) op compiler, plan_dual_sweeps, on random
//       unitary circuits with Pauli-generated parametric gates at 3 and 4
//       register bits: its ops, interpreted by a host restatement of the
//       two-store tile pass, give every derivative sum and both final states
//       of the gates applied one by one
//   engine_host_check halfchains
//       fuse_half_chains on random op lists of two sweeps: runs of
//       half-diagonals on one register bit become pending factors (ACC) and
//       one application (D2HP) inside a sweep, never across sweeps, and the
//       fused list gives every register group the unfused list's result
#include "engine.cpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>

static int check_headers() {
    const int C = 8;
    const uint32_t cshift = 4;  // 16 chunks per block
    int bad = 0;
    for (uint64_t nchunks : {64ull, 1ull << 18}) {
        std::vector<qs::ChunkMeta> m(nchunks);
        std::vector<uint8_t> mask(nchunks >> cshift, 1);
        uint64_t off = 0;
        for (uint64_t k = 0; k < nchunks; ++k) {
            m[k] = qs::ChunkMeta{off, 5, (uint32_t)(k % 33)};
            off += qs::payload_bytes(C, (uint32_t)(k % 33));
        }
        auto chk = [&] { return store_headers_valid(mask.data(), (const char *)m.data(), nchunks, cshift, C, off); };
        const uint64_t j = nchunks - 3;
        const qs::ChunkMeta save = m[j];
        bad += !chk();
        m[j].offset += 8;
        bad += chk();
        m[j] = save;
        m[j].width = 40;
        bad += chk();
        m[j] = save;
        m[j].offset = off;
        m[j].width = 1;
        bad += chk();
        m[j] = save;
        mask[j >> cshift] = 0;
        m[j].offset = 7;
        m[j].width = 99;
        bad += !chk();
    }
    printf("headers: %d failures\n", bad);
    return bad == 0 ? 0 : 1;
}

static int check_plan(const char *path, uint32_t n, uint32_t B, uint32_t I, bool f64) {
    FILE *f = fopen(path, "rb");
    if (!f) return 2;
    uint64_t cnt = 0;
    if (fread(&cnt, 8, 1, f) != 1) return 2;
    std::vector<qs_gate> g(cnt);
    if (fread(g.data(), sizeof(qs_gate), cnt, f) != cnt) return 2;
    fclose(f);
    qs_state h;
    h.n = n;
    h.B = B;
    h.C = std::min<uint32_t>(B, (uint32_t)qs::kMaxChunkLog2);
    h.nb = 1u << (n - B);
    h.nchunks = uint64_t(1) << (n - h.C);
    h.f64 = f64;
    h.tile_log2 = std::min<int>(std::max<int>(f64 ? 12 : 13, (int)h.C + 2),
                                std::min<int>(qs::kMaxTileLog2, (int)h.C + qs::kMaxTileQubits));
    h.gates = g;
    h.cgates.resize(cnt);
    for (size_t i = 0; i < cnt; ++i) {
        std::string e;
        if (!canonicalize(g[i], false, n, &h.cgates[i], &e)) {
            printf("canonicalize: %s\n", e.c_str());
            return 2;
        }
    }
    h.stages = partition_circuit(&h, I);
    make_block_groups(&h);
    HostPlan plan;
    if (plan_device_passes(&h, &plan) != QS_OK) {
        printf("plan: %s\n", h.err.c_str());
        return 2;
    }
    const int jmax = std::min(h.tile_log2 - (int)h.C, qs::kMaxTileQubits);
    for (const auto &dp : h.passes)
        printf("pass kind %d j %d codes %d jmax %d\n", dp.kind, dp.j, dp.code_moves ? 1 : 0, jmax);
    printf("passes %zu\n", h.passes.size());
    return 0;
}

// Plans every stage and, for each start stage s0, the merged tail of stages
// [s0, end): prints the per-stage passes from s0 on, the tail's passes and
// the tail pass that ends each stage.
static int check_tail(const char *path, uint32_t n, uint32_t B, uint32_t I, bool f64) {
    FILE *f = fopen(path, "rb");
    if (!f) return 2;
    uint64_t cnt = 0;
    if (fread(&cnt, 8, 1, f) != 1) return 2;
    std::vector<qs_gate> g(cnt);
    if (fread(g.data(), sizeof(qs_gate), cnt, f) != cnt) return 2;
    fclose(f);
    qs_state h;
    h.n = n;
    h.B = B;
    h.C = std::min<uint32_t>(B, (uint32_t)env_int("QOMPSIM_CHUNK_LOG2", qs::kMaxChunkLog2));
    h.nb = 1u << (n - B);
    h.nchunks = uint64_t(1) << (n - h.C);
    h.f64 = f64;
    h.tile_log2 = std::min<int>(std::max<int>(f64 ? 12 : 13, (int)h.C + 2),
                                std::min<int>(qs::kMaxTileLog2, (int)h.C + qs::kMaxTileQubits));
    h.gates = g;
    h.cgates.resize(cnt);
    for (size_t i = 0; i < cnt; ++i) {
        std::string e;
        if (!canonicalize(g[i], false, n, &h.cgates[i], &e)) return 2;
    }
    h.stages = partition_circuit(&h, I);
    make_block_groups(&h);
    HostPlan plan;
    if (plan_device_passes(&h, &plan) != QS_OK) return 2;
    for (uint32_t s0 = 0; s0 + 1 < h.stages.size(); ++s0) {
        size_t per_stage = 0;
        for (const auto &dp : h.passes) per_stage += dp.stage >= s0 ? 1 : 0;
        HostPlan tp;
        std::vector<qs_state::DevPass> passes;
        std::vector<int> ends;
        if (plan_tail_passes(&h, s0, &tp, &passes, &ends) != QS_OK) return 2;
        printf("tail %u per_stage %zu merged %zu ends", s0, per_stage, passes.size());
        for (int e : ends) printf(" %d", e);
        printf("\n");
    }
    return 0;
}

// The two device rules for an op's variant (rop_variant in kernels.cu):
// selector bit j of the variant is bit sel[j] of the word W, or, with the
// run encoding, runs [a, a + la) and [b, b + lb) of W side by side.
static uint32_t variant_per_bit(const qs::ROp &o, uint32_t W) {
    uint32_t v = 0;
    for (int j = 0; j < o.nsel; ++j) v |= ((W >> o.sel[j]) & 1u) << j;
    return v;
}
static uint32_t variant_from_runs(const qs::ROp &o, uint32_t W) {
    const uint32_t a = o.sel[0] & 31u, la = o.sel[1], b = o.sel[2], lb = o.sel[3];
    return ((W >> a) & ((1u << la) - 1u)) | (((W >> b) & ((1u << lb) - 1u)) << la);
}

static int check_selruns() {
    std::mt19937 rng(7);
    int bad = 0, encoded = 0, kept = 0;
    for (int t = 0; t < 4000; ++t) {
        const int ns = 1 + (int)(rng() % qs::kMaxSel);
        std::vector<int> pos;
        if (rng() % 2) {
            // one or two runs of consecutive bits below bit 31
            const int len1 = 1 + (int)(rng() % ns), len2 = ns - len1;
            const int s1 = (int)(rng() % (31 - ns));
            for (int k = 0; k < len1; ++k) pos.push_back(s1 + k);
            if (len2) {
                const int room = 31 - (s1 + len1 + 1) - len2;
                const int s2 = s1 + len1 + 1 + (room > 0 ? (int)(rng() % (room + 1)) : 0);
                for (int k = 0; k < len2; ++k) pos.push_back(s2 + k);
            }
        } else {
            std::vector<int> all(31);
            for (int k = 0; k < 31; ++k) all[k] = k;
            std::shuffle(all.begin(), all.end(), rng);
            pos.assign(all.begin(), all.begin() + ns);
        }
        std::shuffle(pos.begin(), pos.end(), rng);  // the variant's bit order is the selector order
        std::vector<int> sorted(pos);
        std::sort(sorted.begin(), sorted.end());
        int runs = 1;
        for (int k = 1; k < ns; ++k) runs += sorted[k] != sorted[k - 1] + 1;
        const int stride = 1 + (int)(rng() % 4);
        qs::ROp o{};
        o.code = qs::OPC_M2;
        o.nsel = (uint8_t)ns;
        o.vstride = (uint8_t)stride;
        for (int j = 0; j < ns; ++j) o.sel[j] = (uint8_t)pos[j];
        o.mat = 3;
        std::vector<cplx> pool(o.mat + ((size_t)1 << ns) * stride);
        for (size_t k = 0; k < pool.size(); ++k) pool[k] = cplx((double)k, (double)t);
        const std::vector<cplx> old(pool);
        const qs::ROp orig = o;
        encode_selector_runs(&o, stride, &pool);
        if (runs <= 2) {
            ++encoded;
            bad += !(o.sel[0] & qs::kSelRuns) || o.mat != orig.mat || o.nsel != orig.nsel;
            for (int w = 0; w < 256 && !bad; ++w) {
                const uint32_t W = (uint32_t)rng() & 0x7fffffffu;
                const uint32_t vr = variant_from_runs(o, W), vb = variant_per_bit(orig, W);
                for (int e = 0; e < stride; ++e)
                    bad += pool[o.mat + (size_t)vr * stride + e] != old[orig.mat + (size_t)vb * stride + e];
            }
        } else {
            ++kept;
            bad += std::memcmp(&o, &orig, sizeof(o)) != 0 || pool != old;
        }
        if (bad) {
            printf("selruns: trial %d (%d selectors, %d runs) failed\n", t, ns, runs);
            return 1;
        }
    }
    printf("selruns ok %d encoded %d kept\n", encoded, kept);
    return encoded > 0 && kept > 0 ? 0 : 1;
}

// The register ops of the check below, restated from apply_rop and the
// r_* helpers in kernels.cu: D2 multiplies element s of the group by d0 or
// d1 according to bit K of s, D2H by d1 where bit K is set, D2HP by zh d1
// there and then resets zh to 1, ACC multiplies zh, M2 mixes every pair of
// elements that differ in bit K, SCALAR multiplies z, which scales the whole
// group once the sweep's ops are done.
static void host_rop(std::vector<cplx> &v, cplx &z, cplx &zh, int code, const cplx *m) {
    const int NS = (int)v.size();
    auto in = [&](int base) { return code >= base && code < base + 8; };
    if (code == qs::OPC_SCALAR) {
        z *= m[0];
    } else if (code == qs::OPC_ACC) {
        zh *= m[0];
    } else if (in(qs::OPC_D2)) {
        const int K = code - qs::OPC_D2;
        for (int t = 0; t < NS; ++t) v[t] *= ((t >> K) & 1) ? m[1] : m[0];
    } else if (in(qs::OPC_D2H)) {
        const int K = code - qs::OPC_D2H;
        for (int t = 0; t < NS; ++t)
            if ((t >> K) & 1) v[t] *= m[0];
    } else if (in(qs::OPC_D2HP)) {
        const int K = code - qs::OPC_D2HP;
        const cplx d = zh * m[0];
        for (int t = 0; t < NS; ++t)
            if ((t >> K) & 1) v[t] *= d;
        zh = cplx(1.0, 0.0);
    } else if (in(qs::OPC_M2)) {
        const int K = code - qs::OPC_M2;
        for (int t = 0; t < NS; ++t) {
            if ((t >> K) & 1) continue;
            const cplx a = v[t], b = v[t | (1 << K)];
            v[t] = m[0] * a + m[1] * b;
            v[t | (1 << K)] = m[2] * a + m[3] * b;
        }
    }
}

static std::vector<cplx> host_sweeps(const std::vector<qs::ROp> &ops, const std::vector<qs::Sweep> &sw,
                                     const std::vector<cplx> &pool, std::vector<cplx> v) {
    for (const auto &w : sw) {
        cplx z(1.0, 0.0), zh(1.0, 0.0);  // per group and sweep, as on the device
        for (int k = w.g0; k < w.g1; ++k) host_rop(v, z, zh, ops[k].code, pool.data() + ops[k].mat);
        for (auto &x : v) x *= z;
    }
    return v;
}

static int check_halfchains() {
    std::mt19937 rng(11);
    std::uniform_real_distribution<double> ang(-3.14159, 3.14159), amp(0.5, 1.5);
    int fused = 0;
    for (int t = 0; t < 3000; ++t) {
        const int nops = 2 + (int)(rng() % 24), split = (int)(rng() % (nops + 1));
        std::vector<qs::ROp> ops;
        std::vector<cplx> pool;
        for (int k = 0; k < nops; ++k) {
            qs::ROp o{};
            const int bit = (int)(rng() % 4), kind = (int)(rng() % 8);
            // mostly half-diagonals on few bits, so that runs form
            const int code = kind < 5 ? qs::OPC_D2H + (int)(rng() % 2) : kind == 5 ? qs::OPC_D2 + bit
                           : kind == 6 ? qs::OPC_M2 + bit : qs::OPC_SCALAR;
            const int nm = code >= qs::OPC_M2 ? 4 : (code >= qs::OPC_D2 && code < qs::OPC_D2H) ? 2 : 1;
            o.code = (uint8_t)code;
            o.vstride = (uint8_t)nm;
            o.mat = (uint32_t)pool.size();
            for (int e = 0; e < nm; ++e) pool.push_back(std::polar(amp(rng), ang(rng)));
            ops.push_back(o);
        }
        std::vector<qs::Sweep> sw(2);
        sw[0] = qs::Sweep{0, split, {0, 1, 2, 3, 0, 0}};
        sw[1] = qs::Sweep{split, nops, {0, 1, 2, 3, 0, 0}};
        std::vector<qs::ROp> f(ops);
        fuse_half_chains(&f, 0, sw);
        for (int k = 0; k < nops; ++k) {
            fused += f[k].code == qs::OPC_ACC;
            // an ACC hands its factor to the next op of its own sweep
            const bool last = k + 1 == split || k + 1 == nops;
            if (f[k].code == qs::OPC_ACC && last) {
                printf("halfchains: trial %d: pending factor at the end of a sweep\n", t);
                return 1;
            }
        }
        for (int g = 0; g < 4; ++g) {
            std::vector<cplx> v(16);
            for (auto &x : v) x = std::polar(amp(rng), ang(rng));
            const auto a = host_sweeps(ops, sw, pool, v), b = host_sweeps(f, sw, pool, v);
            for (int e = 0; e < 16; ++e)
                if (std::abs(a[e] - b[e]) > 1e-12 * (1.0 + std::abs(a[e]))) {
                    printf("halfchains: trial %d: element %d differs (%g)\n", t, e, std::abs(a[e] - b[e]));
                    return 1;
                }
        }
    }
    printf("halfchains ok %d fused\n", fused);
    return fused > 0 ? 0 : 1;
}

static int check_dagplan() {
    std::mt19937 rng(5);
    long pairs = 0, moved = 0;
    for (int t = 0; t < 2000; ++t) {
        const int C = 4 + (int)(rng() % 5), n = C + 2 + (int)(rng() % 24);
        const int jmax = 3 + (int)(rng() % 3), jmin = jmax;
        const int G = 1 + (int)(rng() % 160);
        std::vector<CGate> cg(G);
        for (auto &g : cg) {
            g.nq = 1 + (int)(rng() % 2);
            g.q[0] = (int)(rng() % n);
            do g.q[1] = (int)(rng() % n); while (g.nq == 2 && g.q[1] == g.q[0]);
            for (int b = 0; b < g.nq; ++b) g.mix[b] = rng() % 2;
        }
        std::vector<uint32_t> ids(G);
        for (int i = 0; i < G; ++i) ids[i] = (uint32_t)i;
        for (int dag = 0; dag < 2; ++dag) {
            const auto pl = dag ? plan_passes_dag(ids, cg, C, jmax, jmin, C, n) : plan_passes(ids, cg, C, jmax, jmin, C, n);
            std::vector<int> pos(G, -1);
            int k = 0;
            for (const auto &p : pl) {
                std::set<int> tile(p.tile.begin(), p.tile.end()), outer;
                if (tile.size() != p.tile.size() || (int)tile.size() > std::max(jmax, jmin)) {
                    printf("dagplan: trial %d: tile of %zu qubits\n", t, p.tile.size());
                    return 1;
                }
                for (uint32_t gi : p.gates) {
                    if (gi >= (uint32_t)G || pos[gi] >= 0) {
                        printf("dagplan: trial %d: gate %u placed twice or unknown\n", t, gi);
                        return 1;
                    }
                    pos[gi] = k++;
                    for (int b = 0; b < cg[gi].nq; ++b) {
                        const int q = cg[gi].q[b];
                        if (q < C) continue;
                        if (cg[gi].mix[b] && !tile.count(q)) {
                            printf("dagplan: trial %d: gate %u mixes qubit %d outside its tile\n", t, gi, q);
                            return 1;
                        }
                        if (!cg[gi].mix[b] && !tile.count(q)) outer.insert(q);
                    }
                }
                if ((int)outer.size() > qs::kMaxOuterSel) {
                    printf("dagplan: trial %d: %zu outer selector qubits\n", t, outer.size());
                    return 1;
                }
            }
            if (k != G) {
                printf("dagplan: trial %d: %d of %d gates placed\n", t, k, G);
                return 1;
            }
            for (int i = 0; i < G; ++i)
                for (int j = i + 1; j < G; ++j) {
                    bool conflict = false;
                    for (int a = 0; a < cg[i].nq; ++a)
                        for (int b = 0; b < cg[j].nq; ++b)
                            conflict |= cg[i].q[a] == cg[j].q[b] && (cg[i].mix[a] || cg[j].mix[b]);
                    if (!conflict) {
                        moved += dag && pos[i] > pos[j];
                        continue;
                    }
                    ++pairs;
                    if (pos[i] > pos[j]) {
                        printf("dagplan: trial %d (%s): gates %d and %d do not commute but changed order\n", t,
                               dag ? "dag" : "linear", i, j);
                        return 1;
                    }
                }
        }
    }
    printf("dagplan ok %ld ordered pairs, %ld commuting pairs reordered\n", pairs, moved);
    return moved > 0 ? 0 : 1;
}

// A gate on a dense vector: index bit i of the matrix (row-major) is qubit q[i].
static void host_apply(std::vector<cplx> &v, const CGate &g) {
    const int dim = 1 << g.nq;
    uint64_t mask = 0;
    for (int i = 0; i < g.nq; ++i) mask |= 1ull << g.q[i];
    for (uint64_t base = 0; base < v.size(); ++base) {
        if (base & mask) continue;
        uint64_t idx[4];
        cplx x[4], y[4];
        for (int c = 0; c < dim; ++c) {
            idx[c] = base;
            for (int i = 0; i < g.nq; ++i)
                if ((c >> i) & 1) idx[c] |= 1ull << g.q[i];
            x[c] = v[idx[c]];
        }
        for (int r = 0; r < dim; ++r) {
            y[r] = 0;
            for (int c = 0; c < dim; ++c) y[r] += g.m[r * dim + c] * x[c];
        }
        for (int r = 0; r < dim; ++r) v[idx[r]] = y[r];
    }
}

// The chunk moves of a pass's output permutation (apply_perm in kernels.cu):
// chunk c goes to c with bit dst[k] taken from bit src[k], the kept bits
// unchanged, then the flip bits flipped.
static uint64_t host_apply_perm(const qs::ChunkPerm &p, uint64_t c) {
    uint64_t o = c & p.keep;
    for (int k = 0; k < p.nmove; ++k) o |= ((c >> p.src[k]) & 1ull) << p.dst[k];
    return o ^ p.flip;
}

// Every register op of a single-store pass on a group of 16 elements,
// restated from apply_rop and the r_* helpers in kernels.cu.  Codes of one
// register bit are BASE + K; codes of two bits are BASE + 8 A + B.
static void host_rop_any(cplx *v, cplx &z, cplx &zh, int code, const cplx *m) {
    const int NS = 1 << qs::kRegBits;
    auto in = [&](int base, int span) { return code >= base && code < base + span; };
    if (code == qs::OPC_SCALAR) {
        z *= m[0];
    } else if (code == qs::OPC_ACC) {
        zh *= m[0];
    } else if (in(qs::OPC_D2, 8) || in(qs::OPC_D2H, 8) || in(qs::OPC_D2HP, 8) || in(qs::OPC_M2, 8) ||
               in(qs::OPC_X, 8)) {
        const int base = code & ~7, K = code & 7;
        cplx d1 = 0;  // X ops carry no matrix entries: m is read only by the others
        if (base == qs::OPC_D2H) d1 = m[0];
        if (base == qs::OPC_D2HP) {
            d1 = zh * m[0];
            zh = cplx(1.0, 0.0);
        }
        for (int t = 0; t < NS; ++t) {
            const bool hi = (t >> K) & 1;
            if (base == qs::OPC_D2) v[t] *= hi ? m[1] : m[0];
            else if ((base == qs::OPC_D2H || base == qs::OPC_D2HP) && hi) v[t] *= d1;
            else if ((base == qs::OPC_M2 || base == qs::OPC_X) && !hi) {
                const cplx a = v[t], b = v[t | (1 << K)];
                v[t] = base == qs::OPC_X ? b : m[0] * a + m[1] * b;
                v[t | (1 << K)] = base == qs::OPC_X ? a : m[2] * a + m[3] * b;
            }
        }
    } else {
        const int base = code >= qs::OPC_SWAP ? qs::OPC_SWAP : code >= qs::OPC_M4 ? qs::OPC_M4
                       : code >= qs::OPC_D4H ? qs::OPC_D4H : qs::OPC_D4;
        const int A = (code - base) >> 3, B = (code - base) & 7;
        for (int t = 0; t < NS; ++t) {
            const int k = ((t >> A) & 1) | (((t >> B) & 1) << 1);
            if (base == qs::OPC_D4) v[t] *= m[k];
            else if (base == qs::OPC_D4H && k) v[t] *= m[k - 1];
        }
        if (base == qs::OPC_M4 || base == qs::OPC_SWAP)
            for (int t = 0; t < NS; ++t) {
                if (((t >> A) & 1) || ((t >> B) & 1)) continue;
                const int i[4] = {t, t | (1 << A), t | (1 << B), t | (1 << A) | (1 << B)};
                const cplx x[4] = {v[i[0]], v[i[1]], v[i[2]], v[i[3]]};
                for (int r = 0; r < 4; ++r) {
                    if (base == qs::OPC_SWAP) {
                        v[i[r]] = x[r == 1 ? 2 : r == 2 ? 1 : r];
                        continue;
                    }
                    cplx acc = 0;
                    for (int c = 0; c < 4; ++c) acc += m[4 * r + c] * x[c];
                    v[i[r]] = acc;
                }
            }
    }
}

// rop_variant in kernels.cu: the op's matrix variant for selector word W.
static uint32_t host_variant(const qs::ROp &o, uint32_t W) {
    if (o.sel[0] & qs::kSelRuns) return variant_from_runs(o, W);
    uint32_t var = 0;
    for (int j = 0; j < o.nsel; ++j) var |= ((W >> o.sel[j]) & 1u) << j;
    return var;
}

static uint64_t host_insert_zero_bits(uint64_t x, const std::vector<int> &pos) {
    for (int t : pos) x = ((x >> t) << (t + 1)) | (x & ((1ull << t) - 1));
    return x;
}

// One fused tile pass over a dense vector, restated from dense_pass_kernel
// and tile_sweeps: tile element e holds chunk element e mod 2^C of the
// chunk whose tile-qubit bits are e >> C; a sweep walks the groups of 16
// elements that differ in its register bits; the selector word is the
// group's first element index with the tile's outer-qubit bits above it.
static void host_tile_pass(std::vector<cplx> &st, int n, int C, const std::vector<int> &tile,
                           const std::vector<qs::Sweep> &sw, const std::vector<qs::ROp> &ops,
                           const std::vector<cplx> &pool, const std::vector<int> &outer) {
    const int j = (int)tile.size(), nb = C + j, RB = qs::kRegBits;
    std::vector<int> tq(j);
    for (int k = 0; k < j; ++k) tq[k] = tile[k] - C;
    std::vector<cplx> t(1ull << nb);
    for (uint64_t tid = 0; tid < (1ull << (n - nb)); ++tid) {
        const uint64_t cb = host_insert_zero_bits(tid, tq);
        auto amp = [&](uint64_t e) {
            uint64_t c = cb;
            for (int k = 0; k < j; ++k) c |= ((e >> (C + k)) & 1ull) << tq[k];
            return (c << C) | (e & ((1ull << C) - 1));
        };
        for (uint64_t e = 0; e < t.size(); ++e) t[e] = st[amp(e)];
        uint32_t ow = 0;
        for (size_t i = 0; i < outer.size(); ++i) ow |= (uint32_t)(((cb << C) >> outer[i]) & 1ull) << i;
        for (const auto &w : sw) {
            std::vector<int> sb(w.sbits, w.sbits + RB);
            for (uint64_t g = 0; g < (1ull << (nb - RB)); ++g) {
                const uint64_t base = host_insert_zero_bits(g, sb);
                const uint32_t W = (uint32_t)base | (ow << nb);
                cplx v[16];
                auto off = [&](int s2) {
                    uint64_t o = 0;
                    for (int k = 0; k < RB; ++k)
                        if ((s2 >> k) & 1) o |= 1ull << sb[k];
                    return o;
                };
                for (int s2 = 0; s2 < 16; ++s2) v[s2] = t[base | off(s2)];
                cplx z(1.0, 0.0), zh(1.0, 0.0);
                for (int k = w.g0; k < w.g1; ++k)
                    host_rop_any(v, z, zh, ops[k].code, pool.data() + ops[k].mat + host_variant(ops[k], W) * ops[k].vstride);
                for (int s2 = 0; s2 < 16; ++s2) t[base | off(s2)] = z * v[s2];
            }
        }
        for (uint64_t e = 0; e < t.size(); ++e) st[amp(e)] = t[e];
    }
}

// Random circuits through the fused path's host steps (plan_passes_dag,
// tiles padded to the register bits, to_kgate, plan_sweeps, build_ops,
// merge_diagonal_ops, finalize_ops, fuse_half_chains, as in
// qs_dense_apply_gates) and then through host_tile_pass, against the gates
// applied one by one.
static int check_opcompile() {
    std::mt19937 rng(17);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const cplx one(1.0, 0.0), zero(0.0, 0.0);
    const int RB = qs::kRegBits;
    long nops = 0, nsel = 0;
    for (int t = 0; t < 400; ++t) {
        const int n = 7 + (int)(rng() % 5), C = 2 + (int)(rng() % 4), jmax = 3 + (int)(rng() % 3);
        const int G = 1 + (int)(rng() % 60);
        std::vector<CGate> cg;
        for (int k = 0; k < G; ++k) {
            CGate g;
            g.nq = 1 + (int)(rng() % 2);
            g.q[0] = (int)(rng() % n);
            do g.q[1] = (int)(rng() % n); while (g.nq == 2 && g.q[1] == g.q[0]);
            if (g.nq == 2 && g.q[0] > g.q[1]) std::swap(g.q[0], g.q[1]);
            const int dim = 1 << g.nq, kind = (int)(rng() % 6);
            for (int e = 0; e < 16; ++e) g.m[e] = zero;
            if (kind == 0) {  // diagonal (phases, controlled phases when one entry differs)
                for (int r = 0; r < dim; ++r) g.m[r * dim + r] = rng() % 2 ? one : std::polar(1.0, u(rng) * 3);
            } else if (kind == 1) {  // permutation: X, SWAP, CNOT
                const int pk = (int)(rng() % 3);
                for (int r = 0; r < dim; ++r) {
                    const int c = dim == 2 ? r ^ 1 : pk == 0 ? (r == 1 ? 2 : r == 2 ? 1 : r) : pk == 1 ? r ^ 3 : (r & 1 ? r ^ 2 : r);
                    g.m[r * dim + c] = one;
                }
            } else if (kind == 2 && dim == 4) {  // block-diagonal: mixes one qubit, selects by the other
                const int sel = (int)(rng() % 2);
                for (int b = 0; b < 2; ++b)
                    for (int r = 0; r < 2; ++r)
                        for (int c = 0; c < 2; ++c) {
                            const int R = sel ? (r | (b << 1)) : (b | (r << 1)), Cc = sel ? (c | (b << 1)) : (b | (c << 1));
                            g.m[R * 4 + Cc] = cplx(u(rng), u(rng));
                        }
            } else {  // dense
                for (int e = 0; e < dim * dim; ++e) g.m[e] = cplx(u(rng), u(rng));
            }
            compute_mixing(&g);
            cg.push_back(g);
        }
        std::vector<cplx> v(1ull << n);
        for (auto &x : v) x = cplx(u(rng), u(rng));
        std::vector<cplx> want(v), got(v);
        for (const auto &g : cg) host_apply(want, g);
        std::vector<uint32_t> ids(G);
        for (int k = 0; k < G; ++k) ids[k] = (uint32_t)k;
        auto pl = plan_passes_dag(ids, cg, C, jmax, std::min(jmax, 3), C, n);
        for (auto &pp : pl) {
            std::set<int> ts(pp.tile.begin(), pp.tile.end());
            for (int q = C; q < n && C + (int)ts.size() < RB; ++q) ts.insert(q);
            pp.tile.assign(ts.begin(), ts.end());
            const int nb = C + (int)pp.tile.size();
            if (nb < RB || nb > n) {
                printf("opcompile: trial %d: tile of %d bits\n", t, nb);
                return 1;
            }
            std::vector<qs::KGate> kg;
            for (uint32_t gi : pp.gates) kg.push_back(to_kgate(cg[gi], pp.tile, C));
            auto swp = plan_sweeps(kg, 0, kg.size(), nb, RB);
            std::vector<RawOp> raw;
            std::vector<cplx> rpool, pool;
            build_ops(kg, 0, swp, RB, &raw, &rpool);
            std::vector<qs::Sweep> merged;
            merge_diagonal_ops(swp, 0, &raw, &rpool, &merged);
            std::vector<int> outer;
            std::vector<qs::ROp> ops;
            if (!finalize_ops(raw, rpool, nb, &outer, &ops, &pool)) {
                printf("opcompile: trial %d: too many outer selectors\n", t);
                return 1;
            }
            fuse_half_chains(&ops, 0, merged);
            nops += (long)ops.size();
            for (const auto &o : ops) nsel += o.nsel;
            host_tile_pass(got, n, C, pp.tile, merged, ops, pool, outer);
        }
        for (uint64_t k = 0; k < want.size(); ++k)
            if (std::abs(got[k] - want[k]) > 1e-9 * (1.0 + std::abs(want[k]))) {
                printf("opcompile: trial %d (n %d, C %d, jmax %d, %d gates, %zu passes): amplitude %llu differs "
                       "(%g vs %g)\n", t, n, C, jmax, G, pl.size(), (unsigned long long)k, std::abs(got[k]),
                       std::abs(want[k]));
                return 1;
            }
    }
    printf("opcompile ok %ld ops, %ld selector bits\n", nops, nsel);
    return 0;
}

// A two-store pass, restated from dual_tile_sweeps: every gate op acts on
// the groups of both stores (each with its own pending scalars), and an
// OPC_SUM op adds f conj(zb) za sum_s conj(w[s ^ xs]) (-1)^{|s & zs|} v[s]
// to its slot (f: the op's +-1 variant for the Z bits outside the group).
static void host_dual_pass(std::vector<cplx> &A, std::vector<cplx> &B, int n, int C, int RB,
                           const std::vector<int> &tile, const qs::Sweep *sw, size_t nsw, const qs::ROp *ops,
                           const std::vector<cplx> &pool, const std::vector<int> &outer, std::vector<cplx> *sums) {
    const int j = (int)tile.size(), nb = C + j, NS = 1 << RB;
    std::vector<int> tq(j);
    for (int k = 0; k < j; ++k) tq[k] = tile[k] - C;
    std::vector<cplx> ta(1ull << nb), tb(1ull << nb);
    for (uint64_t tid = 0; tid < (1ull << (n - nb)); ++tid) {
        const uint64_t cb = host_insert_zero_bits(tid, tq);
        auto amp = [&](uint64_t e) {
            uint64_t c = cb;
            for (int k = 0; k < j; ++k) c |= ((e >> (C + k)) & 1ull) << tq[k];
            return (c << C) | (e & ((1ull << C) - 1));
        };
        for (uint64_t e = 0; e < ta.size(); ++e) {
            ta[e] = A[amp(e)];
            tb[e] = B[amp(e)];
        }
        uint32_t ow = 0;
        for (size_t i = 0; i < outer.size(); ++i) ow |= (uint32_t)(((cb << C) >> outer[i]) & 1ull) << i;
        for (size_t si = 0; si < nsw; ++si) {
            const qs::Sweep &w = sw[si];
            std::vector<int> sb(w.sbits, w.sbits + RB);
            auto off = [&](int s2) {
                uint64_t o = 0;
                for (int k = 0; k < RB; ++k)
                    if ((s2 >> k) & 1) o |= 1ull << sb[k];
                return o;
            };
            for (uint64_t g = 0; g < (1ull << (nb - RB)); ++g) {
                const uint64_t base = host_insert_zero_bits(g, sb);
                const uint32_t W = (uint32_t)base | (ow << nb);
                // the interpreter works on 16-element groups; with RB = 3 the
                // upper half stays zero and no op of the sweep touches bit 3
                cplx v[16] = {}, u[16] = {};
                for (int s2 = 0; s2 < NS; ++s2) {
                    v[s2] = ta[base | off(s2)];
                    u[s2] = tb[base | off(s2)];
                }
                cplx za(1.0, 0.0), zb(1.0, 0.0), zha(1.0, 0.0), zhb(1.0, 0.0);
                for (int k = w.g0; k < w.g1; ++k) {
                    const qs::ROp &o = ops[k];
                    if (o.code == qs::OPC_SUM) {
                        const int xs = o.pad >> 4, zs = o.pad & 15;
                        cplx acc = 0;
                        for (int s2 = 0; s2 < NS; ++s2)
                            acc += std::conj(u[s2 ^ xs]) * v[s2] * ((__builtin_popcount(s2 & zs) & 1) ? -1.0 : 1.0);
                        (*sums)[o.vstride] += pool[o.mat + host_variant(o, W)] * std::conj(zb) * za * acc;
                    } else {
                        const cplx *m = pool.data() + o.mat + host_variant(o, W) * o.vstride;
                        host_rop_any(v, za, zha, o.code, m);
                        host_rop_any(u, zb, zhb, o.code, m);
                    }
                }
                for (int s2 = 0; s2 < NS; ++s2) {
                    ta[base | off(s2)] = za * v[s2];
                    tb[base | off(s2)] = zb * u[s2];
                }
            }
        }
        for (uint64_t e = 0; e < ta.size(); ++e) {
            A[amp(e)] = ta[e];
            B[amp(e)] = tb[e];
        }
    }
}

// A random unitary of size dim (Gram-Schmidt on random complex columns):
// the adjoint's sums are invariant under gates that commute with a
// parametric gate only when those gates are unitary.
static void random_unitary(int dim, cplx *m, std::mt19937 &rng) {
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (int c = 0; c < dim; ++c) {
        cplx col[4];
        for (int r = 0; r < dim; ++r) col[r] = cplx(u(rng), u(rng));
        for (int p = 0; p < c; ++p) {
            cplx d = 0;
            for (int r = 0; r < dim; ++r) d += std::conj(m[r * dim + p]) * col[r];
            for (int r = 0; r < dim; ++r) col[r] -= d * m[r * dim + p];
        }
        double nrm = 0;
        for (int r = 0; r < dim; ++r) nrm += std::norm(col[r]);
        nrm = std::sqrt(nrm);
        for (int r = 0; r < dim; ++r) m[r * dim + c] = col[r] / nrm;
    }
}

// plan_dual_sweeps on random circuits with parametric gates: the two-store
// ops, interpreted by host_dual_pass, give for each parametric gate
// sum_x conj(B[x ^ gx]) (-1)^{|x & gz|} A[x] taken just before the gate,
// and the states of every gate applied to both stores one by one.
static int check_dualcompile() {
    std::mt19937 rng(19);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const cplx one(1.0, 0.0), zero(0.0, 0.0);
    long nsum = 0, fused_passes = 0, passes = 0;
    for (int t = 0; t < 300; ++t) {
        const int RB = t % 2 ? qs::kDualRegBitsF32 : qs::kDualRegBitsF64;
        const int n = 7 + (int)(rng() % 4), C = 2 + (int)(rng() % 4), jmax = 3 + (int)(rng() % 3);
        const int G = 1 + (int)(rng() % 40);
        std::vector<CGate> cg;
        std::vector<int32_t> slots(G, -1);
        std::vector<uint64_t> gx(G, 0), gz(G, 0);
        int nslot = 0;
        for (int k = 0; k < G; ++k) {
            CGate g;
            g.nq = 1 + (int)(rng() % 2);
            g.q[0] = (int)(rng() % n);
            do g.q[1] = (int)(rng() % n); while (g.nq == 2 && g.q[1] == g.q[0]);
            if (g.nq == 2 && g.q[0] > g.q[1]) std::swap(g.q[0], g.q[1]);
            const int dim = 1 << g.nq;
            for (int e = 0; e < 16; ++e) g.m[e] = zero;
            if (rng() % 3 == 0)
                for (int r = 0; r < dim; ++r) g.m[r * dim + r] = std::polar(1.0, u(rng) * 3);
            else
                random_unitary(dim, g.m, rng);
            compute_mixing(&g);
            if (rng() % 2) {  // parametric: a Pauli generator on the gate's own qubits
                slots[k] = nslot++;
                for (int b = 0; b < g.nq; ++b) {
                    const int pk = (int)(rng() % 4);  // I, X, Y, Z
                    if (pk == 1 || pk == 2) gx[k] |= 1ull << g.q[b];
                    if (pk == 2 || pk == 3) gz[k] |= 1ull << g.q[b];
                    if (pk == 1 || pk == 2) g.mix[b] = true;  // as qs_dense_adjoint: flipped qubits mix
                }
            }
            cg.push_back(g);
        }
        // reference: every gate on both stores in order, each sum just before its gate
        std::vector<cplx> a0(1ull << n), b0(1ull << n);
        for (auto &x : a0) x = cplx(u(rng), u(rng));
        for (auto &x : b0) x = cplx(u(rng), u(rng));
        std::vector<cplx> wa(a0), wb(b0), want(nslot, 0.0);
        for (int k = 0; k < G; ++k) {
            if (slots[k] >= 0)
                for (uint64_t x = 0; x < wa.size(); ++x)
                    want[slots[k]] += std::conj(wb[x ^ gx[k]]) * wa[x] * ((__builtin_popcountll(x & gz[k]) & 1) ? -1.0 : 1.0);
            host_apply(wa, cg[k]);
            host_apply(wb, cg[k]);
        }
        std::vector<cplx> ga(a0), gb(b0), got(nslot, 0.0);
        std::vector<uint32_t> ids(G);
        for (int k = 0; k < G; ++k) ids[k] = (uint32_t)k;
        auto pl = plan_passes_dag(ids, cg, C, jmax, std::min(jmax, 3), C, n);
        for (auto &pp : pl) {
            std::set<int> ts(pp.tile.begin(), pp.tile.end());
            for (int q = C; q < n && C + (int)ts.size() < RB; ++q) ts.insert(q);
            pp.tile.assign(ts.begin(), ts.end());
            std::vector<qs::Sweep> asw;
            std::vector<qs::ROp> arops;
            std::vector<cplx> apool;
            DualSweepPlan dp;
            ++passes;
            if (!plan_dual_sweeps(cg, pp.gates, slots.data(), gx.data(), gz.data(), pp.tile, C, RB, &asw, &arops,
                                  &apool, &dp)) {
                // not fusable: the engine runs such a pass op by op; here the reference steps stand in
                for (uint32_t gi : pp.gates) {
                    if (slots[gi] >= 0)
                        for (uint64_t x = 0; x < ga.size(); ++x)
                            got[slots[gi]] += std::conj(gb[x ^ gx[gi]]) * ga[x] *
                                              ((__builtin_popcountll(x & gz[gi]) & 1) ? -1.0 : 1.0);
                    host_apply(ga, cg[gi]);
                    host_apply(gb, cg[gi]);
                }
                continue;
            }
            ++fused_passes;
            std::vector<cplx> local(std::max(1, nslot), 0.0);
            host_dual_pass(ga, gb, n, C, RB, pp.tile, asw.data() + dp.sw_off, dp.nsw, arops.data() + dp.rop_off, apool,
                           dp.outer, &local);
            int ls = 0;
            for (uint32_t gi : pp.gates)
                if (slots[gi] >= 0) {
                    got[slots[gi]] += local[ls++];
                    ++nsum;
                }
        }
        double scale = 1.0;
        for (const auto &x : wa) scale = std::max(scale, std::abs(x));
        for (const auto &x : wb) scale = std::max(scale, std::abs(x));
        // |sum| <= |A| |B|, both norms kept by the unitary gates
        double na = 0, nb2 = 0;
        for (const auto &x : a0) na += std::norm(x);
        for (const auto &x : b0) nb2 += std::norm(x);
        const double tol = 1e-12 * std::sqrt(na * nb2) * (1 + G);
        for (int k = 0; k < nslot; ++k)
            if (std::abs(got[k] - want[k]) > tol) {
                printf("dualcompile: trial %d (RB %d, n %d, C %d): sum %d differs (%g vs %g)\n", t, RB, n, C, k,
                       std::abs(got[k]), std::abs(want[k]));
                return 1;
            }
        for (uint64_t x = 0; x < wa.size(); ++x)
            if (std::abs(ga[x] - wa[x]) > 1e-9 * scale || std::abs(gb[x] - wb[x]) > 1e-9 * scale) {
                printf("dualcompile: trial %d (RB %d): amplitude %llu differs\n", t, RB, (unsigned long long)x);
                return 1;
            }
    }
    printf("dualcompile ok %ld of %ld passes fused, %ld sums\n", fused_passes, passes, nsum);
    return fused_passes > passes / 2 && nsum > 0 ? 0 : 1;
}

static int check_chunkperm() {
    std::mt19937 rng(13);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const cplx one(1.0, 0.0), zero(0.0, 0.0);
    int folded = 0;
    for (int t = 0; t < 2000; ++t) {
        const int n = 6 + (int)(rng() % 5), C = 2 + (int)(rng() % 3), G = 1 + (int)(rng() % 40);
        std::vector<CGate> cg;
        for (int k = 0; k < G; ++k) {
            CGate g;
            const int kind = (int)(rng() % 6);
            g.nq = kind == 1 || kind == 3 ? 1 : 2;
            const bool high = kind <= 1 || kind == 5;  // SWAP / X / X x X on qubits >= C
            const int lo = high ? C : 0;
            g.q[0] = lo + (int)(rng() % (n - lo));
            do g.q[1] = lo + (int)(rng() % (n - lo)); while (g.nq == 2 && g.q[1] == g.q[0]);
            if (g.nq == 2 && g.q[0] > g.q[1]) std::swap(g.q[0], g.q[1]);
            const int dim = 1 << g.nq;
            for (int e = 0; e < 16; ++e) g.m[e] = zero;
            if (kind == 0) {         // SWAP
                g.m[0] = g.m[1 * 4 + 2] = g.m[2 * 4 + 1] = g.m[15] = one;
            } else if (kind == 1) {  // X
                g.m[1] = g.m[2] = one;
            } else if (kind == 5) {  // X on both qubits
                for (int r = 0; r < 4; ++r) g.m[r * 4 + (r ^ 3)] = one;
            } else if (kind == 4 && rng() % 2) {  // CNOT: a permutation that is not folded
                g.m[0] = g.m[1 * 4 + 3] = g.m[2 * 4 + 2] = g.m[3 * 4 + 1] = one;
            } else if (rng() % 3 == 0) {          // diagonal
                for (int r = 0; r < dim; ++r) g.m[r * dim + r] = cplx(u(rng), u(rng));
            } else {                              // dense
                for (int e = 0; e < dim * dim; ++e) g.m[e] = cplx(u(rng), u(rng));
            }
            compute_mixing(&g);
            cg.push_back(g);
        }
        std::vector<uint32_t> ids(G);
        for (int k = 0; k < G; ++k) ids[k] = (uint32_t)k;
        std::vector<CGate> out;
        HostPerm P(n - C);
        stage_relabel(cg, ids, C, true, &out, &P);
        folded += G - (int)out.size();
        std::vector<cplx> v(1ull << n);
        for (auto &x : v) x = cplx(u(rng), u(rng));
        std::vector<cplx> want(v), got(v);
        for (const auto &g : cg) host_apply(want, g);
        for (const auto &g : out) host_apply(got, g);
        const qs::ChunkPerm dp = P.device();
        std::vector<cplx> moved(got.size());
        const uint64_t cm = (1ull << C) - 1;
        for (uint64_t k = 0; k < got.size(); ++k) moved[(host_apply_perm(dp, k >> C) << C) | (k & cm)] = got[k];
        for (uint64_t k = 0; k < want.size(); ++k)
            if (std::abs(moved[k] - want[k]) > 1e-9 * (1.0 + std::abs(want[k]))) {
                printf("chunkperm: trial %d (n %d, C %d, %d gates): amplitude %llu differs\n", t, n, C, G,
                       (unsigned long long)k);
                return 1;
            }
    }
    printf("chunkperm ok %d gates folded\n", folded);
    return folded > 0 ? 0 : 1;
}

int main(int argc, char **argv) {
    if (argc > 1 && !strcmp(argv[1], "selruns")) return check_selruns();
    if (argc > 1 && !strcmp(argv[1], "chunkperm")) return check_chunkperm();
    if (argc > 1 && !strcmp(argv[1], "opcompile")) return check_opcompile();
    if (argc > 1 && !strcmp(argv[1], "dualcompile")) return check_dualcompile();
    if (argc > 1 && !strcmp(argv[1], "dagplan")) return check_dagplan();
    if (argc > 1 && !strcmp(argv[1], "halfchains")) return check_halfchains();
    if (argc > 1 && !strcmp(argv[1], "headers")) return check_headers();
    if (argc > 6 && !strcmp(argv[1], "plan"))
        return check_plan(argv[2], (uint32_t)atoi(argv[3]), (uint32_t)atoi(argv[4]), (uint32_t)atoi(argv[5]),
                          atoi(argv[6]) != 0);
    if (argc > 6 && !strcmp(argv[1], "tail"))
        return check_tail(argv[2], (uint32_t)atoi(argv[3]), (uint32_t)atoi(argv[4]), (uint32_t)atoi(argv[5]),
                          atoi(argv[6]) != 0);
    return 2;
}
