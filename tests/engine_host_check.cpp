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

int main(int argc, char **argv) {
    if (argc > 1 && !strcmp(argv[1], "headers")) return check_headers();
    if (argc > 6 && !strcmp(argv[1], "plan"))
        return check_plan(argv[2], (uint32_t)atoi(argv[3]), (uint32_t)atoi(argv[4]), (uint32_t)atoi(argv[5]),
                          atoi(argv[6]) != 0);
    if (argc > 6 && !strcmp(argv[1], "tail"))
        return check_tail(argv[2], (uint32_t)atoi(argv[3]), (uint32_t)atoi(argv[4]), (uint32_t)atoi(argv[5]),
                          atoi(argv[6]) != 0);
    return 2;
}
