// ref_pf_flop_mats — test infrastructure: runs the reference's own
// kernel_gen_100_flop_matrices and kernel_reduce_combo_to_class_matrices
// (src/preflop/preflop_grid_generator.cu:128-223) for a few subset flops,
// compiled from the reference's source file by oracle/Makefile (target `ref`,
// with the reference's --use_fast_math, output in oracle/_ref/), and writes
// the class-reduced equity matrices.
//
// Inputs as preflop_gen builds them (:468-502): the combos are the first 1,176
// pairs c1 < c2 in lexicographic order, and each class lists, in that order,
// up to 12 of its combos.  The caller passes each combo's class (the
// reference's class numbering).  The combo-matrix buffer is zeroed before the
// generator runs: the generator leaves the entries of hero combos that touch
// the flop unwritten, and the reduction reads them (and skips entries that are
// not above 0).  Only the two kernels above are launched; their grids
// (1,176 x count and 169 x count) and the [count][1216][1216] and
// [count][169][169] buffers cover every index they form, and each hero's
// local deck holds exactly the 47 cards off the flop and the hero's hand.
//
// Input (little-endian): int32 count; count SubsetFlop records (c1, c2, c3,
// pad, f32 weight; cards distinct); int16 class[1176].
// Output: class matrices [count][169][169] (f32), [flop][villain][hero].
//
// usage: ref_pf_flop_mats in.bin out.bin
#define main mtt_reference_stub_main
#include "preflop_grid_generator.cu"
#undef main

#include <cstdio>

static bool read_exact(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_pf_flop_mats in.bin out.bin\n");
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int32_t count = 0;
    if (!read_exact(f, &count, 4) || count < 1 || count > 100) return 2;   // the generator's grid check is f < 100
    std::vector<SubsetFlop> subset(count);
    std::vector<int16_t> cls(N_ALIVE_COMBOS);
    if (!read_exact(f, subset.data(), sizeof(SubsetFlop) * count) || !read_exact(f, cls.data(), 2 * cls.size())) return 1;
    std::fclose(f);
    for (const SubsetFlop& s : subset)
        if (s.c1 > 51 || s.c2 > 51 || s.c3 > 51 || s.c1 == s.c2 || s.c1 == s.c3 || s.c2 == s.c3) return 2;
    std::vector<AliveCombo> alive(N_PADDED_COMBOS, AliveCombo{0, 0, 0});
    std::vector<ClassComboList> lists(N_CLASSES);
    for (auto& l : lists) { l.count = 0; for (auto& x : l.combo_idx) x = 0; }
    int n = 0;
    for (int c1 = 0; c1 < 52 && n < (int)N_ALIVE_COMBOS; ++c1)
        for (int c2 = c1 + 1; c2 < 52 && n < (int)N_ALIVE_COMBOS; ++c2, ++n) {
            alive[n] = AliveCombo{(uint8_t)c1, (uint8_t)c2, (1ull << c1) | (1ull << c2)};
            const int k = cls[n];
            if (k < 0 || k >= (int)N_CLASSES) return 2;
            if (lists[k].count < 12) lists[k].combo_idx[lists[k].count++] = (uint16_t)n;
        }
    SubsetFlop* d_subset;
    AliveCombo* d_combos;
    ClassComboList* d_lists;
    float *d_combo_mats, *d_class_mats;
    const size_t n_combo = (size_t)count * N_PADDED_COMBOS * N_PADDED_COMBOS, n_class = (size_t)count * N_CLASSES * N_CLASSES;
    CUDA_CHECK(cudaMalloc(&d_subset, sizeof(SubsetFlop) * count));
    CUDA_CHECK(cudaMalloc(&d_combos, sizeof(AliveCombo) * alive.size()));
    CUDA_CHECK(cudaMalloc(&d_lists, sizeof(ClassComboList) * lists.size()));
    CUDA_CHECK(cudaMalloc(&d_combo_mats, sizeof(float) * n_combo));
    CUDA_CHECK(cudaMalloc(&d_class_mats, sizeof(float) * n_class));
    CUDA_CHECK(cudaMemcpy(d_subset, subset.data(), sizeof(SubsetFlop) * count, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_combos, alive.data(), sizeof(AliveCombo) * alive.size(), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_lists, lists.data(), sizeof(ClassComboList) * lists.size(), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemset(d_combo_mats, 0, sizeof(float) * n_combo));
    CUDA_CHECK(cudaMemset(d_class_mats, 0, sizeof(float) * n_class));
    kernel_gen_100_flop_matrices<<<dim3((unsigned)N_ALIVE_COMBOS, (unsigned)count), 256>>>(d_subset, d_combos, d_combo_mats);
    CUDA_CHECK(cudaGetLastError());
    kernel_reduce_combo_to_class_matrices<<<dim3((unsigned)N_CLASSES, (unsigned)count), 256>>>(count, d_combo_mats, d_lists,
                                                                                            d_class_mats);
    CUDA_CHECK(cudaGetLastError());
    CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<float> out(n_class);
    CUDA_CHECK(cudaMemcpy(out.data(), d_class_mats, sizeof(float) * n_class, cudaMemcpyDeviceToHost));
    FILE* w = std::fopen(argv[2], "wb");
    if (!w) return 1;
    bool ok = std::fwrite(out.data(), sizeof(float), n_class, w) == n_class;
    ok = (std::fclose(w) == 0) && ok;
    return ok ? 0 : 1;
}
