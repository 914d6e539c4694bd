// preflop_gen — drop-in for the reference's preflop_gen
// (src/preflop/preflop_grid_generator.cu:426-653): reads the flop subset
// (data/mtt_subset.bin, then ./mtt_subset.bin), builds the 169 x 169 all-in
// matrix and the class-reduced flop matrices, runs the preflop DCFR and prints
// the 15-hand BTN / BB strategy table.
#include <chrono>
#include <iomanip>
#include <iostream>

#include "driver_util.h"

int main(int argc, char** argv) {
    const char* subset = nullptr;
    int mode = MTT_PF_REFERENCE;
    mtt_pf_params p = {500, 20.0f, 1.35f, 2.5f};
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() { return i + 1 < argc ? argv[++i] : ""; };
        if (a == "--subset") subset = val();
        else if (a == "--mode") mode = std::string(val()) == "correct" ? MTT_PF_CORRECT : MTT_PF_REFERENCE;
        else if (a == "--iters") p.iters = std::atoi(val());
        else if (a == "--stack") p.stack_bb = (float)std::atof(val());
        else if (a == "--bubble") p.bubble = (float)std::atof(val());
        else if (a == "--dead") p.dead_pot = (float)std::atof(val());
        else {
            std::cout << "usage: preflop_gen [--subset FILE] [--mode reference|correct] [--iters 500] [--stack 20]"
                         " [--bubble 1.35] [--dead 2.5]\n";
            return a == "--help" || a == "-h" ? 0 : 1;
        }
    }
    int32_t n = 0;
    if (mtt_pf_read_subset(subset, nullptr, nullptr, 0, &n) != MTT_OK || n <= 0) {
        std::cerr << "cannot read the flop subset (data/mtt_subset.bin or ./mtt_subset.bin)\n";
        return 1;
    }
    std::vector<uint8_t> flops(3 * (size_t)n);
    std::vector<float> w(n);
    DRV_CHECK(mtt_pf_read_subset(subset, flops.data(), w.data(), n, &n));
    std::cout << "Loaded " << n << " flops\n";
    uint8_t* d_flops = nullptr;
    float *d_w = nullptr, *d_allin = nullptr, *d_mats = nullptr, *d_sums = nullptr, *d_sig = nullptr;
    DRV_CUDA(cudaMalloc(&d_flops, flops.size()));
    DRV_CUDA(cudaMalloc(&d_w, sizeof(float) * n));
    DRV_CUDA(cudaMalloc(&d_allin, sizeof(float) * 169 * 169));
    DRV_CUDA(cudaMalloc(&d_mats, sizeof(float) * 169 * 169 * (size_t)n));
    DRV_CUDA(cudaMalloc(&d_sums, sizeof(float) * 10 * 192));
    DRV_CUDA(cudaMalloc(&d_sig, sizeof(float) * 10 * 192));
    DRV_CUDA(cudaMemcpy(d_flops, flops.data(), flops.size(), cudaMemcpyHostToDevice));
    DRV_CUDA(cudaMemcpy(d_w, w.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    const auto t0 = std::chrono::steady_clock::now();
    DRV_CHECK(mtt_pf_allin_matrix(mode, d_allin, nullptr, nullptr, nullptr));
    DRV_CHECK(mtt_pf_flop_class_matrices(mode, d_flops, n, d_mats, nullptr));
    DRV_CUDA(cudaDeviceSynchronize());
    const auto t1 = std::chrono::steady_clock::now();
    DRV_CHECK(mtt_pf_dcfr(d_w, d_mats, n, d_allin, &p, d_sums, d_sig, nullptr));
    DRV_CUDA(cudaDeviceSynchronize());
    const auto t2 = std::chrono::steady_clock::now();
    const double ms_m = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const double ms_d = std::chrono::duration<double, std::milli>(t2 - t1).count();
    std::cout << "    Matrices in " << ms_m / 1000.0 << " s\n";
    std::cout << "    DCFR Loop Done in " << ms_d / 1000.0 << " s (" << p.iters / (ms_d / 1000.0) << " iter/sec)\n";
    std::vector<float> sums(10 * 192);
    DRV_CUDA(cudaMemcpy(sums.data(), d_sums, sizeof(float) * sums.size(), cudaMemcpyDeviceToHost));
    // the reference's display hands and their class indices
    const char* names[15] = {"AA", "KK", "QQ", "JJ", "TT", "99", "88", "22", "AKs", "A5s", "T9s", "76s", "AKo", "QJo", "32o"};
    const int idx[15] = {0, 1, 2, 3, 4, 5, 6, 12, 13, 17, 72, 85, 91, 104, 168};
    const std::string rule(88, '=');
    std::cout << "\n" << rule << "\n  GTO SNAPSHOT: " << p.stack_bb << " BB (BF = " << p.bubble << ") BTN vs BB ("
              << (mode == MTT_PF_REFERENCE ? "reference" : "correct") << " mode)\n" << rule << "\n";
    std::cout << std::left << std::setw(7) << "Hand" << std::setw(12) << "BTN Fold" << std::setw(14) << "BTN MinRaise"
              << std::setw(12) << "BTN Jam" << std::setw(12) << "BB Fold" << std::setw(14) << "BB Defend"
              << std::setw(12) << "BB 3B-Jam" << "\n" << std::string(88, '-') << "\n";
    for (int i = 0; i < 15; ++i) {
        const int c = idx[i];
        float b[3], d[3];
        for (int a = 0; a < 3; ++a) { b[a] = sums[(0 + a) * 192 + c]; d[a] = sums[(3 + a) * 192 + c]; }
        const float tb = b[0] + b[1] + b[2] + 1e-7f, td = d[0] + d[1] + d[2] + 1e-7f;
        std::cout << std::left << std::setw(7) << names[i] << std::fixed << std::setprecision(3) << std::setw(12)
                  << b[0] / tb << std::setw(14) << b[1] / tb << std::setw(12) << b[2] / tb << std::setw(12) << d[0] / td
                  << std::setw(14) << d[1] / td << std::setw(12) << d[2] / td << "\n";
    }
    std::cout << rule << "\n";
    cudaFree(d_flops); cudaFree(d_w); cudaFree(d_allin); cudaFree(d_mats); cudaFree(d_sums); cudaFree(d_sig);
    return 0;
}
