// subset_optimizer — drop-in for the reference's scripts/optimize_subset.py.
// Reads mtt_ev_dump_1755.bin from the working directory (or --dump PATH),
// selects --select flops (100 by default) by greedy non-negative orthogonal
// matching pursuit on the device (mtt_subset_nnomp) and writes mtt_subset.bin
// and mtt_subset_weights.txt to the working directory in the reference's
// formats (optimize_subset.py:52-65).
#include <fstream>
#include <iostream>

#include "driver_util.h"

int main(int argc, char** argv) {
    std::string dump_path = "mtt_ev_dump_1755.bin";
    int nselect = 100;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--dump") && i + 1 < argc) dump_path = argv[++i];
        else if (!std::strcmp(argv[i], "--select") && i + 1 < argc) nselect = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--help") || !std::strcmp(argv[i], "-h")) {
            std::cout << "usage: subset_optimizer [--dump PATH] [--select N]   "
                         "(writes mtt_subset.bin and mtt_subset_weights.txt)\n";
            return 0;
        } else {
            std::cerr << "unknown argument " << argv[i] << "\n";
            return 2;
        }
    }
    const int nfeat = 4 * 2 * 169;
    std::vector<uint8_t> fl(4 * 1755);
    int32_t n = 0;
    DRV_CHECK(mtt_canonical_flops(fl.data(), 1755, &n));
    std::vector<float> dump((size_t)n * nfeat);
    {
        std::ifstream f(dump_path, std::ios::binary);
        f.read(reinterpret_cast<char*>(dump.data()), (std::streamsize)(dump.size() * sizeof(float)));
        if (!f || f.gcount() != (std::streamsize)(dump.size() * sizeof(float))) {
            std::cerr << "cannot read " << dump.size() << " floats from " << dump_path << "\n";
            return 1;
        }
    }
    std::vector<double> colw(n);
    for (int j = 0; j < n; ++j) colw[j] = fl[4 * j + 3];
    float* d_cols = nullptr;
    double *d_colw = nullptr, *d_w = nullptr;
    int32_t* d_idx = nullptr;
    DRV_CUDA(cudaMalloc(&d_cols, sizeof(float) * dump.size()));
    DRV_CUDA(cudaMalloc(&d_colw, sizeof(double) * n));
    DRV_CUDA(cudaMalloc(&d_w, sizeof(double) * std::max(nselect, 1)));
    DRV_CUDA(cudaMalloc(&d_idx, sizeof(int32_t) * std::max(nselect, 1)));
    DRV_CUDA(cudaMemcpy(d_cols, dump.data(), sizeof(float) * dump.size(), cudaMemcpyHostToDevice));
    DRV_CUDA(cudaMemcpy(d_colw, colw.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    DRV_CHECK(mtt_subset_nnomp(d_cols, n, nfeat, d_colw, nselect, d_idx, d_w, nullptr));
    std::vector<int32_t> idx(nselect);
    std::vector<double> w(nselect);
    DRV_CUDA(cudaMemcpy(idx.data(), d_idx, sizeof(int32_t) * nselect, cudaMemcpyDeviceToHost));
    DRV_CUDA(cudaMemcpy(w.data(), d_w, sizeof(double) * nselect, cudaMemcpyDeviceToHost));
    std::vector<uint8_t> f3;
    for (int i = 0; i < nselect; ++i)
        for (int k = 0; k < 3; ++k) f3.push_back(fl[4 * idx[i] + k]);
    DRV_CHECK(mtt_subset_write("mtt_subset.bin", "mtt_subset_weights.txt", f3.data(), w.data(), nselect));
    cudaFree(d_cols);
    cudaFree(d_colw);
    cudaFree(d_w);
    cudaFree(d_idx);
    std::cout << "Subset generated: " << nselect << " flops saved to mtt_subset.bin\n";
    return 0;
}
