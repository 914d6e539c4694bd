// ref_pf_dcfr — test infrastructure: runs the reference's own preflop DCFR
// loop, kernel_update_dynamic_reaches / kernel_cosolve_100_board_matrices /
// kernel_build_closed_preflop_cfvs / kernel_dcfr_step
// (src/preflop/preflop_grid_generator.cu:228-421), with its host loop's
// schedule and initial state (:545-614), compiled from the reference's source
// file by oracle/Makefile (target `ref`, with the reference's --use_fast_math,
// output in oracle/_ref/).
//
// The matrices the loop reads are inputs: the all-in equity matrix and the
// class-reduced flop matrices in the reference's layouts.  The reference's own
// all-in kernel (kernel_gen_preflop_matrix) is not run: it writes past its
// local deck[48] array when a sampled hand repeats a card.  Only the four
// loop kernels above are launched; each indexes [169] or [192] class rows
// and the [count][169][169] matrices with a class index below 169.
//
// Input (little-endian): int32 count, iters; f32 stack_bb, bubble, dead_pot;
// count SubsetFlop records (c1, c2, c3, pad, f32 weight); class matrices
// [count][169][169] f32; all-in matrix [169][169] f32.
// Output: strategy sums [10][192] then last strategies [10][192] (f32): rows
// 0-2 BTN root, 3-5 BB defence, 6-7 BTN vs 3-bet jam, 8-9 BB vs open jam.
//
// usage: ref_pf_dcfr in.bin out.bin
#define main mtt_reference_stub_main
#include "preflop_grid_generator.cu"
#undef main

#include <cstdio>

static bool read_exact(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: ref_pf_dcfr in.bin out.bin\n");
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 1;
    int32_t hdr[2];
    float par[3];
    if (!read_exact(f, hdr, 8) || !read_exact(f, par, 12)) return 1;
    const int count = hdr[0], iters = hdr[1];
    if (count < 1 || count > 100000 || iters < 1 || iters > 1000000) return 2;
    const float stack_bb = par[0], bf = par[1], dead_pot = par[2];
    std::vector<SubsetFlop> subset(count);
    std::vector<float> mats((size_t)count * N_CLASSES * N_CLASSES), allin(N_CLASSES * N_CLASSES);
    if (!read_exact(f, subset.data(), sizeof(SubsetFlop) * subset.size()) ||
        !read_exact(f, mats.data(), sizeof(float) * mats.size()) || !read_exact(f, allin.data(), sizeof(float) * allin.size()))
        return 1;
    std::fclose(f);
    SubsetFlop* d_subset;
    float *d_mats, *d_allin;
    CUDA_CHECK(cudaMalloc(&d_subset, sizeof(SubsetFlop) * count));
    CUDA_CHECK(cudaMalloc(&d_mats, sizeof(float) * mats.size()));
    CUDA_CHECK(cudaMalloc(&d_allin, sizeof(float) * allin.size()));
    CUDA_CHECK(cudaMemcpy(d_subset, subset.data(), sizeof(SubsetFlop) * count, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_mats, mats.data(), sizeof(float) * mats.size(), cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_allin, allin.data(), sizeof(float) * allin.size(), cudaMemcpyHostToDevice));
    // the state of the reference's host loop (:545-578)
    const size_t act3 = 3 * N_CLASSES_PADDED * 4, a2 = 2 * N_CLASSES_PADDED * 4, a1 = N_CLASSES_PADDED * 4;
    float *d_r_btn, *d_s_btn, *d_sums_btn, *d_cfv_btn, *d_r_bb, *d_s_bb, *d_sums_bb, *d_cfv_bb;
    float *d_r_btn_3b, *d_s_btn_3b, *d_sums_btn_3b, *d_cfv_btn_3b, *d_r_bb_jam, *d_s_bb_jam, *d_sums_bb_jam, *d_cfv_bb_jam;
    float *d_root_reach_btn, *d_root_reach_bb, *d_reach_btn_call, *d_reach_bb_call, *d_flop_net_ev_btn, *d_flop_net_ev_bb;
    for (float** p : {&d_r_btn, &d_s_btn, &d_sums_btn, &d_cfv_btn, &d_r_bb, &d_s_bb, &d_sums_bb, &d_cfv_bb})
        CUDA_CHECK(cudaMalloc(p, act3));
    for (float** p : {&d_r_btn_3b, &d_s_btn_3b, &d_sums_btn_3b, &d_cfv_btn_3b, &d_r_bb_jam, &d_s_bb_jam, &d_sums_bb_jam,
                      &d_cfv_bb_jam})
        CUDA_CHECK(cudaMalloc(p, a2));
    for (float** p : {&d_root_reach_btn, &d_root_reach_bb, &d_reach_btn_call, &d_reach_bb_call, &d_flop_net_ev_btn,
                      &d_flop_net_ev_bb}) {
        CUDA_CHECK(cudaMalloc(p, a1));
        CUDA_CHECK(cudaMemset(*p, 0, a1));
    }
    for (float** p : {&d_cfv_btn, &d_cfv_bb}) CUDA_CHECK(cudaMemset(*p, 0, act3));
    for (float** p : {&d_cfv_btn_3b, &d_cfv_bb_jam}) CUDA_CHECK(cudaMemset(*p, 0, a2));
    CUDA_CHECK(cudaMemset(d_r_btn, 0, act3)); CUDA_CHECK(cudaMemset(d_sums_btn, 0, act3));
    CUDA_CHECK(cudaMemset(d_r_bb, 0, act3)); CUDA_CHECK(cudaMemset(d_sums_bb, 0, act3));
    CUDA_CHECK(cudaMemset(d_r_btn_3b, 0, a2)); CUDA_CHECK(cudaMemset(d_sums_btn_3b, 0, a2));
    CUDA_CHECK(cudaMemset(d_r_bb_jam, 0, a2)); CUDA_CHECK(cudaMemset(d_sums_bb_jam, 0, a2));
    std::vector<float> init_3(3 * N_CLASSES_PADDED, 1.0f / 3.0f), init_2(2 * N_CLASSES_PADDED, 0.5f);
    CUDA_CHECK(cudaMemcpy(d_s_btn, init_3.data(), act3, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_s_bb, init_3.data(), act3, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_s_btn_3b, init_2.data(), a2, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_s_bb_jam, init_2.data(), a2, cudaMemcpyHostToDevice));
    std::vector<float> init_r(N_CLASSES_PADDED, 0.0f);
    for (size_t i = 0; i < N_CLASSES; ++i) init_r[i] = (i < 13 ? 6.0f : (i < 91 ? 4.0f : 12.0f)) / 1326.0f;
    CUDA_CHECK(cudaMemcpy(d_root_reach_btn, init_r.data(), a1, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(d_root_reach_bb, init_r.data(), a1, cudaMemcpyHostToDevice));
    dim3 block(128), grid((N_CLASSES + block.x - 1) / block.x);
    for (int t = 1; t <= iters; ++t) {   // :588-614
        const float tf = static_cast<float>(t);
        const float wp = powf(tf, 1.5f) / (powf(tf, 1.5f) + 1.0f);
        const float ws = tf * tf;
        kernel_update_dynamic_reaches<<<grid, block>>>(d_root_reach_btn, d_root_reach_bb, d_s_btn, d_s_bb,
                                                       d_reach_btn_call, d_reach_bb_call);
        kernel_cosolve_100_board_matrices<<<grid, block>>>(count, d_subset, d_reach_btn_call, d_reach_bb_call, d_mats,
                                                           d_flop_net_ev_btn, d_flop_net_ev_bb, dead_pot + 3.1f, bf);
        kernel_build_closed_preflop_cfvs<<<grid, block>>>(d_flop_net_ev_btn, d_flop_net_ev_bb, d_s_btn, d_s_bb, d_s_btn_3b,
                                                          d_s_bb_jam, d_root_reach_btn, d_root_reach_bb, d_allin, d_cfv_btn,
                                                          d_cfv_bb, d_cfv_btn_3b, d_cfv_bb_jam, dead_pot, stack_bb, bf);
        kernel_dcfr_step<<<grid, block>>>(3, d_r_btn, d_s_btn, d_sums_btn, d_cfv_btn, d_root_reach_btn, wp, ws);
        kernel_dcfr_step<<<grid, block>>>(3, d_r_bb, d_s_bb, d_sums_bb, d_cfv_bb, d_root_reach_bb, wp, ws);
        kernel_dcfr_step<<<grid, block>>>(2, d_r_btn_3b, d_s_btn_3b, d_sums_btn_3b, d_cfv_btn_3b, d_root_reach_btn, wp, ws);
        kernel_dcfr_step<<<grid, block>>>(2, d_r_bb_jam, d_s_bb_jam, d_sums_bb_jam, d_cfv_bb_jam, d_root_reach_bb, wp, ws);
        CUDA_CHECK(cudaGetLastError());
    }
    CUDA_CHECK(cudaDeviceSynchronize());
    std::vector<float> out(2 * 10 * N_CLASSES_PADDED);
    float* o = out.data();
    const size_t P = N_CLASSES_PADDED;
    CUDA_CHECK(cudaMemcpy(o, d_sums_btn, act3, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(o + 3 * P, d_sums_bb, act3, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(o + 6 * P, d_sums_btn_3b, a2, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(o + 8 * P, d_sums_bb_jam, a2, cudaMemcpyDeviceToHost));
    o += 10 * P;
    CUDA_CHECK(cudaMemcpy(o, d_s_btn, act3, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(o + 3 * P, d_s_bb, act3, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(o + 6 * P, d_s_btn_3b, a2, cudaMemcpyDeviceToHost));
    CUDA_CHECK(cudaMemcpy(o + 8 * P, d_s_bb_jam, a2, cudaMemcpyDeviceToHost));
    FILE* w = std::fopen(argv[2], "wb");
    if (!w) return 1;
    bool ok = std::fwrite(out.data(), sizeof(float), out.size(), w) == out.size();
    ok = (std::fclose(w) == 0) && ok;
    return ok ? 0 : 1;
}
