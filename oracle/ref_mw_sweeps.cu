// ref_mw_sweeps — test infrastructure: runs the reference's own four-player
// CFR+ kernels, kernel_4way_forward_sweep / kernel_4way_evaluate_terminals /
// kernel_4way_backward_cfr_plus (src/postflop/multiway_4way_engine.cu:41-257),
// compiled from the reference's source file by oracle/Makefile (target `ref`,
// output in oracle/_ref/), on a four-player river tree, and writes the
// regrets, strategy sums and root counterfactual values after a number of
// iterations.
//
// The terminal kernel ranks hands by combo_rank_pos, a position per combo
// slot.  The reference's four-player file has no evaluator, so the caller
// passes each live hand's 7-card score on the river board.  The harness
// orders the hands by score with ties in combo order (a stable sort) and gives
// the padding slots the positions after them, so the positions are a
// permutation of 0 .. 1215 and every shared-memory slot the kernel scans is
// written.  Its CTA is 256 threads (CHUNK_SIZE 5 x 256 >= 1216 slots, eight
// warp sums); the sweeps use 256-thread CTAs over the 1,216 slots.
//
// Host loop per iteration t = 1 .. iters, as the kernels imply: forward sweep
// by depth from the root, the terminals, backward sweep by depth to the root
// with iter_weight = t.
//
// Input (little-endian): int32 n_nodes, H, iters, n_infosets; n_nodes FlatNode
// records (32 B; infoset_offset is the node's infoset id); score[H] (u32);
// range[4][H] (f32); bubble factors [4][4] (f32).
// Output: R[n_infosets*3][1216], S[n_infosets*3][1216], root cfv [4][1216] (f32).
//
// usage: ref_mw_sweeps in.bin out.bin
#define main mtt_reference_stub_main
#include "multiway_4way_engine.cu"
#undef main

#include <cstdio>
#include <cstdlib>
#include <numeric>

static_assert(sizeof(FlatNode) == 32, "FlatNode is 32 bytes");

static bool read_exact(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_mw_sweeps in.bin out.bin\n");
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int32_t hdr[4];
    if (!read_exact(f, hdr, sizeof(hdr))) return 1;
    const int n_nodes = hdr[0], H = hdr[1], iters = hdr[2], n_inf = hdr[3];
    if (n_nodes < 1 || n_nodes > 1000000 || H < 1 || H > (int)N_ALIVE_COMBOS || iters < 1 || iters > 100000 ||
        n_inf < 0 || n_inf > n_nodes) {
        std::fprintf(stderr, "bad header\n");
        return 2;
    }
    std::vector<FlatNode> nodes(n_nodes);
    std::vector<uint32_t> score(H);
    std::vector<float> range(N_PLAYERS * (size_t)H), bubble(16);
    if (!read_exact(f, nodes.data(), sizeof(FlatNode) * nodes.size()) ||
        !read_exact(f, score.data(), sizeof(uint32_t) * score.size()) ||
        !read_exact(f, range.data(), sizeof(float) * range.size()) || !read_exact(f, bubble.data(), 64))
        return 1;
    std::fclose(f);
    // check every index the kernels will form against the buffers
    std::vector<int> depth(n_nodes, -1);
    depth[0] = 0;
    int max_depth = 0;
    for (int i = 0; i < n_nodes; ++i) {
        const FlatNode& n = nodes[i];
        if (depth[i] < 0) { std::fprintf(stderr, "node %d unreachable before its index\n", i); return 2; }
        if (n.type == NODE_DECISION) {
            if (n.num_actions < 1 || n.num_actions > (int)MAX_POST_ACTIONS || n.player >= N_PLAYERS ||
                n.children_offset <= i || n.children_offset + n.num_actions > n_nodes || n.infoset_offset < 0 ||
                n.infoset_offset >= n_inf) {
                std::fprintf(stderr, "bad decision node %d\n", i);
                return 2;
            }
            for (int a = 0; a < n.num_actions; ++a) depth[n.children_offset + a] = depth[i] + 1;
            max_depth = std::max(max_depth, depth[i] + 1);
        } else if (n.type == NODE_FOLD_TERMINAL) {
            if ((n.active_mask & 0xF) == 0) { std::fprintf(stderr, "fold %d has no winner\n", i); return 2; }
        } else if (n.type != NODE_SHOWDOWN_TERMINAL) {
            std::fprintf(stderr, "node %d: only decision, fold and showdown nodes\n", i);
            return 2;
        }
    }
    std::vector<std::vector<int>> levels(max_depth + 1);
    std::vector<int> terms;
    for (int i = 0; i < n_nodes; ++i) {
        levels[depth[i]].push_back(i);
        if (nodes[i].type == NODE_FOLD_TERMINAL || nodes[i].type == NODE_SHOWDOWN_TERMINAL) terms.push_back(i);
    }
    // rank positions: live hands by score, ties in combo order; padding after them
    std::vector<int> ord(H);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return score[a] < score[b]; });
    std::vector<uint16_t> pos(N_PADDED_COMBOS);
    for (int k = 0; k < H; ++k) pos[ord[k]] = (uint16_t)k;
    for (int s = H; s < (int)N_PADDED_COMBOS; ++s) pos[s] = (uint16_t)s;
    const size_t P = N_PADDED_COMBOS, NI = (size_t)std::max(n_inf, 1) * MAX_POST_ACTIONS * P;
    FlatNode* d_nodes; uint16_t* d_pos;
    float *d_bf, *d_R, *d_S, *d_sigma, *d_reach, *d_cfv;
    int *d_lv, *d_terms;
    CUDA_CHECK(cudaMalloc(&d_nodes, sizeof(FlatNode) * n_nodes));
    CUDA_CHECK(cudaMalloc(&d_pos, sizeof(uint16_t) * P));
    CUDA_CHECK(cudaMalloc(&d_bf, 64));
    CUDA_CHECK(cudaMalloc(&d_R, sizeof(float) * NI));
    CUDA_CHECK(cudaMalloc(&d_S, sizeof(float) * NI));
    CUDA_CHECK(cudaMalloc(&d_sigma, sizeof(float) * NI));
    CUDA_CHECK(cudaMalloc(&d_reach, sizeof(float) * (size_t)n_nodes * N_PLAYERS * P));
    CUDA_CHECK(cudaMalloc(&d_cfv, sizeof(float) * (size_t)n_nodes * N_PLAYERS * P));
    CUDA_CHECK(cudaMalloc(&d_lv, sizeof(int) * n_nodes));
    CUDA_CHECK(cudaMalloc(&d_terms, sizeof(int) * std::max<size_t>(terms.size(), 1)));
    CUDA_CHECK(cudaMemcpy(d_nodes, nodes.data(), sizeof(FlatNode) * n_nodes, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_pos, pos.data(), sizeof(uint16_t) * P, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_bf, bubble.data(), 64, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_R, 0, sizeof(float) * NI));
    CUDA_CHECK(cudaMemset(d_S, 0, sizeof(float) * NI));
    CUDA_CHECK(cudaMemset(d_sigma, 0, sizeof(float) * NI));
    CUDA_CHECK(cudaMemset(d_reach, 0, sizeof(float) * (size_t)n_nodes * N_PLAYERS * P));
    CUDA_CHECK(cudaMemset(d_cfv, 0, sizeof(float) * (size_t)n_nodes * N_PLAYERS * P));
    for (int p = 0; p < (int)N_PLAYERS; ++p)   // root reach
        CUDA_CHECK(cudaMemcpy(d_reach + p * P, range.data() + (size_t)p * H, sizeof(float) * H, cudaMemcpyHostToDevice));
    if (!terms.empty()) CUDA_CHECK(cudaMemcpy(d_terms, terms.data(), sizeof(int) * terms.size(), cudaMemcpyHostToDevice));
    std::vector<int> flat, off;
    for (auto& l : levels) { off.push_back((int)flat.size()); flat.insert(flat.end(), l.begin(), l.end()); }
    CUDA_CHECK(cudaMemcpy(d_lv, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice));
    const unsigned sweep_blocks = (unsigned)((P + 255) / 256);
    for (int t = 1; t <= iters; ++t) {
        for (int d = 0; d <= max_depth; ++d) {
            const int nd = (int)levels[d].size();
            kernel_4way_forward_sweep<<<dim3(sweep_blocks, nd), 256>>>(d_lv + off[d], nd, d_nodes, d_R, d_sigma, d_reach);
        }
        if (!terms.empty())
            kernel_4way_evaluate_terminals<<<(unsigned)terms.size(), 256>>>(d_terms, (int)terms.size(), d_nodes, d_reach,
                                                                             d_pos, d_bf, d_cfv);
        for (int d = max_depth; d >= 0; --d) {
            const int nd = (int)levels[d].size();
            kernel_4way_backward_cfr_plus<<<dim3(sweep_blocks, nd), 256>>>(d_lv + off[d], nd, d_nodes, d_sigma, d_reach,
                                                                            d_cfv, d_R, d_S, (float)t);
        }
        CUDA_CHECK(cudaGetLastError());
    }
    CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<float> R(NI), S(NI), cfv(N_PLAYERS * P);
    CUDA_CHECK(cudaMemcpy(R.data(), d_R, sizeof(float) * NI, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(S.data(), d_S, sizeof(float) * NI, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(cfv.data(), d_cfv, sizeof(float) * N_PLAYERS * P, cudaMemcpyDeviceToHost));   // root
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 1;
    const size_t nR = (size_t)n_inf * MAX_POST_ACTIONS * P;
    bool ok = std::fwrite(R.data(), sizeof(float), nR, o) == nR && std::fwrite(S.data(), sizeof(float), nR, o) == nR &&
              std::fwrite(cfv.data(), sizeof(float), N_PLAYERS * P, o) == N_PLAYERS * P;
    ok = (std::fclose(o) == 0) && ok;
    return ok ? 0 : 1;
}
