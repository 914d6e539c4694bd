// ref_turn_matrices — test infrastructure: runs the reference's own
// kernel_gen_49_turn_matrices (src/postflop/honest_multistreet_solver.cu:56-86),
// compiled from the reference's source file by oracle/Makefile (target `ref`,
// output in oracle/_ref/), for one flop, and writes its output to a file:
// [49 turns][1216 villain slots][1216 hero slots] f32, each entry the hero's
// equity (wins + ties / 2) / rivers against that villain after that turn.
//
// Inputs as the reference's kernel expects them: the deck is the 49 cards not
// on the flop in increasing order (turn t = deck[t]); the combos are the
// 1,176 pairs c1 < c2 of deck cards in lexicographic order, with their card
// masks.  The buffer is exactly the kernel's [49][1216][1216]; the grid is
// (1176, 49), so every index the kernel forms is inside it.
//
// usage: ref_turn_matrices c1 c2 c3 out.f32
#define main mtt_reference_stub_main
#include "honest_multistreet_solver.cu"
#undef main

#include <cstdio>
#include <cstdlib>

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: ref_turn_matrices c1 c2 c3 out.f32\n");
        return 2;
    }
    int flop[3];
    uint64_t fm = 0;
    for (int k = 0; k < 3; ++k) {
        flop[k] = std::atoi(argv[1 + k]);
        if (flop[k] < 0 || flop[k] > 51 || (fm >> flop[k]) & 1ull) {
            std::fprintf(stderr, "flop cards must be 3 distinct values in 0..51\n");
            return 2;
        }
        fm |= 1ull << flop[k];
    }
    std::vector<uint8_t> deck;
    for (int c = 0; c < 52; ++c)
        if (!((fm >> c) & 1ull)) deck.push_back((uint8_t)c);
    std::vector<AliveCombo> combos;
    for (size_t a = 0; a < deck.size(); ++a)
        for (size_t b = a + 1; b < deck.size(); ++b)
            combos.push_back(AliveCombo{deck[a], deck[b], (1ull << deck[a]) | (1ull << deck[b])});
    if (deck.size() != 49 || combos.size() != N_ALIVE_COMBOS) return 1;
    const uint8_t f8[3] = {(uint8_t)flop[0], (uint8_t)flop[1], (uint8_t)flop[2]};
    const size_t n_out = 49 * N_PADDED_COMBOS * N_PADDED_COMBOS;
    AliveCombo* d_combos = nullptr;
    uint8_t *d_deck = nullptr, *d_flop = nullptr;
    float* d_out = nullptr;
    CUDA_CHECK(cudaMalloc(&d_combos, sizeof(AliveCombo) * combos.size()));
    CUDA_CHECK(cudaMalloc(&d_deck, deck.size()));
    CUDA_CHECK(cudaMalloc(&d_flop, 3));
    CUDA_CHECK(cudaMalloc(&d_out, sizeof(float) * n_out));
    CUDA_CHECK(cudaMemcpy(d_combos, combos.data(), sizeof(AliveCombo) * combos.size(), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_deck, deck.data(), deck.size(), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_flop, f8, 3, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_out, 0xFF, sizeof(float) * n_out));   // NaN where the kernel writes nothing
    kernel_gen_49_turn_matrices<<<dim3((unsigned)N_ALIVE_COMBOS, 49), 128>>>(d_combos, d_deck, d_flop, d_out);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<float> h(n_out);
    CUDA_CHECK(cudaMemcpy(h.data(), d_out, sizeof(float) * n_out, cudaMemcpyDeviceToHost));
    FILE* f = std::fopen(argv[4], "wb");
    if (!f || std::fwrite(h.data(), sizeof(float), n_out, f) != n_out) {
        std::fprintf(stderr, "cannot write %s\n", argv[4]);
        return 1;
    }
    std::fclose(f);
    cudaFree(d_combos);
    cudaFree(d_deck);
    cudaFree(d_flop);
    cudaFree(d_out);
    return 0;
}
