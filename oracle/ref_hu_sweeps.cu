// ref_hu_sweeps — test infrastructure: runs the reference's own heads-up CFR+
// kernels, kernel_forward_sweep / kernel_evaluate_terminals /
// kernel_backward_sweep (src/postflop/honest_multistreet_solver.cu:88-249),
// compiled from the reference's source file by oracle/Makefile (target `ref`,
// output in oracle/_ref/), on a river tree, and writes the regrets, strategy
// sums and root counterfactual values after a number of iterations.
//
// The kernels' showdown reads an equity matrix per turn card.  On a river tree
// there is one board, so the harness passes one [1216][1216] matrix (villain-
// major, as the reference's): 1, 0.5 or 0 for hero against villain on that
// board by the reference's own evaluator, and 0 where the two hands share a
// card (the reference's turn matrices hold 0 there too).  Every showdown node
// reads it (turn_idx 0).  The tree has no chance node.
//
// Launches: the sweeps use 256-thread CTAs over the 1,216 padded combos.  The
// terminal kernel reduces a fold's opponent mass inside one CTA, so it runs
// with 1,024-thread CTAs and the caller keeps every live hand below combo
// 1,024: the first CTA then sums the whole mass.
//
// Host loop per iteration t = 1 .. iters, as the kernels imply: forward sweep
// by depth from the root, the terminals, backward sweep by depth to the root
// with iter_weight = t (linear averaging).
//
// Input (little-endian): int32 n_nodes, H, iters, n_infosets; n_nodes FlatNode
// records (32 B; infoset_offset is the node's infoset id, 0 .. n_infosets-1);
// H hands (c1, c2); 5 board cards; range0[H], range1[H] (f32).
// Output: R[n_infosets*3][1216], S[n_infosets*3][1216], root cfv [2][1216] (f32).
//
// With a third argument `time`, the harness first runs min(iters, 3) warm-up
// iterations, resets the state, then times the `iters` iterations with CUDA
// events on the launching stream and prints "iters_ms <ms> launches <n>".
//
// usage: ref_hu_sweeps in.bin out.bin [time]
#define main mtt_reference_stub_main
#include "honest_multistreet_solver.cu"
#undef main

#include <cstdio>
#include <cstdlib>
#include <cstring>

static_assert(sizeof(FlatNode) == 32, "FlatNode is 32 bytes");

// The river-board equity matrix: eq[j][h] for hero h against villain j.
__global__ void harness_river_equity(const AliveCombo* __restrict__ combos, int H, const uint8_t* __restrict__ board,
                                     float* __restrict__ eq) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (h >= (int)N_PADDED_COMBOS || j >= (int)N_PADDED_COMBOS) return;
    float v = 0.0f;
    if (h < H && j < H && (combos[h].mask & combos[j].mask) == 0) {
        uint8_t h7[7] = {board[0], board[1], board[2], board[3], board[4], combos[h].c1, combos[h].c2};
        uint8_t v7[7] = {board[0], board[1], board[2], board[3], board[4], combos[j].c1, combos[j].c2};
        const uint32_t sh = eval_7cards_fast(h7), sv = eval_7cards_fast(v7);
        v = sh > sv ? 1.0f : (sh == sv ? 0.5f : 0.0f);
    }
    eq[(size_t)j * N_PADDED_COMBOS + h] = v;
}

static bool read_exact(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

int main(int argc, char** argv) {
    if (argc != 3 && !(argc == 4 && std::strcmp(argv[3], "time") == 0)) {
        std::fprintf(stderr, "usage: ref_hu_sweeps in.bin out.bin [time]\n");
        return 2;
    }
    const bool timing = argc == 4;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int32_t hdr[4];
    if (!read_exact(f, hdr, sizeof(hdr))) return 1;
    const int n_nodes = hdr[0], H = hdr[1], iters = hdr[2], n_inf = hdr[3];
    if (n_nodes < 1 || n_nodes > 1000000 || H < 1 || H > 1024 || iters < 1 || iters > 100000 || n_inf < 0 ||
        n_inf > n_nodes) {
        std::fprintf(stderr, "bad header\n");
        return 2;
    }
    std::vector<FlatNode> nodes(n_nodes);
    std::vector<uint8_t> hands(2 * (size_t)H), board(5);
    std::vector<float> range(2 * (size_t)H);
    if (!read_exact(f, nodes.data(), sizeof(FlatNode) * nodes.size()) || !read_exact(f, hands.data(), hands.size()) ||
        !read_exact(f, board.data(), 5) || !read_exact(f, range.data(), sizeof(float) * range.size()))
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
            if (n.num_actions < 1 || n.num_actions > (int)MAX_ACTIONS || n.children_offset <= i ||
                n.children_offset + n.num_actions > n_nodes || n.infoset_offset < 0 || n.infoset_offset >= n_inf) {
                std::fprintf(stderr, "bad decision node %d\n", i);
                return 2;
            }
            for (int a = 0; a < n.num_actions; ++a) depth[n.children_offset + a] = depth[i] + 1;
            max_depth = std::max(max_depth, depth[i] + 1);
        } else if (n.type == NODE_SHOWDOWN_TERMINAL) {
            if (n.turn_idx != 0) { std::fprintf(stderr, "showdown %d: turn_idx must be 0\n", i); return 2; }
        } else if (n.type != NODE_FOLD_TERMINAL) {
            std::fprintf(stderr, "node %d: only decision, fold and showdown nodes\n", i);
            return 2;
        }
    }
    for (int c : board)
        if (c > 51) return 2;
    std::vector<std::vector<int>> levels(max_depth + 1);
    std::vector<int> terms;
    for (int i = 0; i < n_nodes; ++i) {
        levels[depth[i]].push_back(i);
        if (nodes[i].type == NODE_FOLD_TERMINAL || nodes[i].type == NODE_SHOWDOWN_TERMINAL) terms.push_back(i);
    }
    std::vector<AliveCombo> combos(N_ALIVE_COMBOS, AliveCombo{0, 0, 0});
    for (int h = 0; h < H; ++h) {
        const uint8_t a = hands[2 * h], b = hands[2 * h + 1];
        if (a > 51 || b > 51 || a == b) return 2;
        combos[h] = AliveCombo{a, b, (1ull << a) | (1ull << b)};
    }
    std::vector<uint8_t> deck(49, 0);   // no chance node reads it
    const size_t P = N_PADDED_COMBOS, NI = (size_t)std::max(n_inf, 1) * MAX_ACTIONS * P;
    FlatNode* d_nodes; AliveCombo* d_combos; uint8_t *d_deck, *d_board;
    float *d_eq, *d_R, *d_S, *d_sigma, *d_reach, *d_cfv;
    int *d_lv, *d_terms;
    CUDA_CHECK(cudaMalloc(&d_nodes, sizeof(FlatNode) * n_nodes));
    CUDA_CHECK(cudaMalloc(&d_combos, sizeof(AliveCombo) * combos.size()));
    CUDA_CHECK(cudaMalloc(&d_deck, 49));
    CUDA_CHECK(cudaMalloc(&d_board, 5));
    CUDA_CHECK(cudaMalloc(&d_eq, sizeof(float) * P * P));
    CUDA_CHECK(cudaMalloc(&d_R, sizeof(float) * NI));
    CUDA_CHECK(cudaMalloc(&d_S, sizeof(float) * NI));
    CUDA_CHECK(cudaMalloc(&d_sigma, sizeof(float) * NI));
    CUDA_CHECK(cudaMalloc(&d_reach, sizeof(float) * (size_t)n_nodes * 2 * P));
    CUDA_CHECK(cudaMalloc(&d_cfv, sizeof(float) * (size_t)n_nodes * 2 * P));
    CUDA_CHECK(cudaMalloc(&d_lv, sizeof(int) * n_nodes));
    CUDA_CHECK(cudaMalloc(&d_terms, sizeof(int) * std::max<size_t>(terms.size(), 1)));
    CUDA_CHECK(cudaMemcpy(d_nodes, nodes.data(), sizeof(FlatNode) * n_nodes, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_combos, combos.data(), sizeof(AliveCombo) * combos.size(), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_deck, deck.data(), 49, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_board, board.data(), 5, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_R, 0, sizeof(float) * NI));
    CUDA_CHECK(cudaMemset(d_S, 0, sizeof(float) * NI));
    CUDA_CHECK(cudaMemset(d_sigma, 0, sizeof(float) * NI));
    CUDA_CHECK(cudaMemset(d_reach, 0, sizeof(float) * (size_t)n_nodes * 2 * P));
    CUDA_CHECK(cudaMemset(d_cfv, 0, sizeof(float) * (size_t)n_nodes * 2 * P));
    CUDA_CHECK(cudaMemcpy(d_reach, range.data(), sizeof(float) * H, cudaMemcpyHostToDevice));             // root, P0
    CUDA_CHECK(cudaMemcpy(d_reach + P, range.data() + H, sizeof(float) * H, cudaMemcpyHostToDevice));     // root, P1
    if (!terms.empty()) CUDA_CHECK(cudaMemcpy(d_terms, terms.data(), sizeof(int) * terms.size(), cudaMemcpyHostToDevice));
    harness_river_equity<<<dim3((unsigned)((P + 255) / 256), (unsigned)P), 256>>>(d_combos, H, d_board, d_eq);
    CUDA_CHECK(cudaGetLastError());
    // the level lists, one after another in d_lv
    std::vector<int> flat, off;
    for (auto& l : levels) { off.push_back((int)flat.size()); flat.insert(flat.end(), l.begin(), l.end()); }
    CUDA_CHECK(cudaMemcpy(d_lv, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice));
    const unsigned sweep_blocks = (unsigned)((P + 255) / 256);
    long long launches = 0;
    auto run = [&](int n_it) {
    for (int t = 1; t <= n_it; ++t) {
        for (int d = 0; d <= max_depth; ++d) {
            const int nd = (int)levels[d].size();
            kernel_forward_sweep<<<dim3(sweep_blocks, nd), 256>>>(d_lv + off[d], nd, d_nodes, d_deck, d_combos, d_R,
                                                                   d_sigma, d_reach);
        }
        if (!terms.empty())
            kernel_evaluate_terminals<<<dim3(2, (unsigned)terms.size()), 1024>>>(d_terms, (int)terms.size(), d_nodes,
                                                                                  d_reach, d_eq, d_cfv);
        for (int d = max_depth; d >= 0; --d) {
            const int nd = (int)levels[d].size();
            kernel_backward_sweep<<<dim3(sweep_blocks, nd), 256>>>(d_lv + off[d], nd, d_nodes, d_deck, d_combos,
                                                                    d_sigma, d_reach, d_cfv, d_R, d_S, (float)t);
        }
        launches += 2 * (max_depth + 1) + (terms.empty() ? 0 : 1);
        CUDA_CHECK(cudaGetLastError());
    }
    };
    if (!timing) {
        run(iters);
    } else {
        run(std::min(iters, 3));   // warm-up (module loading, clocks), then the same start state again
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaMemset(d_R, 0, sizeof(float) * NI));
        CUDA_CHECK(cudaMemset(d_S, 0, sizeof(float) * NI));
        CUDA_CHECK(cudaMemset(d_sigma, 0, sizeof(float) * NI));
        CUDA_CHECK(cudaMemset(d_cfv, 0, sizeof(float) * (size_t)n_nodes * 2 * P));
        launches = 0;
        cudaEvent_t e0, e1;
        CUDA_CHECK(cudaEventCreate(&e0));
        CUDA_CHECK(cudaEventCreate(&e1));
        CUDA_CHECK(cudaEventRecord(e0, 0));
        run(iters);
        CUDA_CHECK(cudaEventRecord(e1, 0));
        CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        std::printf("iters_ms %.6f launches %lld\n", ms, launches);
    }
    CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<float> R(NI), S(NI), cfv(2 * P);
    CUDA_CHECK(cudaMemcpy(R.data(), d_R, sizeof(float) * NI, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(S.data(), d_S, sizeof(float) * NI, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(cfv.data(), d_cfv, sizeof(float) * 2 * P, cudaMemcpyDeviceToHost));   // node 0 = root
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 1;
    const size_t nR = (size_t)n_inf * MAX_ACTIONS * P;
    bool ok = std::fwrite(R.data(), sizeof(float), nR, o) == nR && std::fwrite(S.data(), sizeof(float), nR, o) == nR &&
              std::fwrite(cfv.data(), sizeof(float), 2 * P, o) == 2 * P;
    ok = (std::fclose(o) == 0) && ok;
    return ok ? 0 : 1;
}
