// ev_dumper — drop-in for the reference's ev_dumper (src/tools/mtt_ev_dumper.cu:118-174).
// Writes mtt_ev_dump_1755.bin to the working directory: little-endian f32
// [flop][4 scenarios][2 players][169 classes] for the first --limit canonical
// flops (all 1,755 by default), bit-exact with the reference.  Flops are split
// across the visible GPUs, one host thread each, as the reference does.
#include <fstream>
#include <iostream>
#include <thread>

#include "driver_util.h"

int main(int argc, char** argv) {
    int limit = 1755;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--limit") && i + 1 < argc) limit = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--help") || !std::strcmp(argv[i], "-h")) {
            std::cout << "usage: ev_dumper [--limit N]   (writes mtt_ev_dump_1755.bin)\n";
            return 0;
        }
    }
    std::vector<uint8_t> fl(4 * 1755);
    int32_t n = 0;
    DRV_CHECK(mtt_canonical_flops(fl.data(), 1755, &n));
    limit = std::max(0, std::min(limit, (int)n));
    const size_t per = 4 * 2 * 169;
    std::vector<float> out((size_t)limit * per, 0.0f);
    int ngpu = 1;
    if (cudaGetDeviceCount(&ngpu) != cudaSuccess || ngpu < 1) ngpu = 1;
    ngpu = std::max(1, std::min(ngpu, limit));
    std::vector<std::thread> th;
    for (int g = 0; g < ngpu && limit > 0; ++g) {
        th.emplace_back([&, g]() {
            const int lo = (int)((long long)limit * g / ngpu), hi = (int)((long long)limit * (g + 1) / ngpu);
            if (hi <= lo) return;
            DRV_CUDA(cudaSetDevice(g));
            std::vector<uint8_t> f3;
            for (int i = lo; i < hi; ++i) for (int k = 0; k < 3; ++k) f3.push_back(fl[4 * i + k]);
            uint8_t* d_f = nullptr;
            float* d_o = nullptr;
            DRV_CUDA(cudaMalloc(&d_f, f3.size()));
            DRV_CUDA(cudaMalloc(&d_o, sizeof(float) * per * (hi - lo)));
            DRV_CUDA(cudaMemcpy(d_f, f3.data(), f3.size(), cudaMemcpyHostToDevice));
            DRV_CHECK(mtt_ev_dump(d_f, hi - lo, d_o, nullptr));
            DRV_CUDA(cudaMemcpy(out.data() + per * lo, d_o, sizeof(float) * per * (hi - lo), cudaMemcpyDeviceToHost));
            cudaFree(d_f);
            cudaFree(d_o);
        });
    }
    for (auto& t : th) t.join();
    std::ofstream f("mtt_ev_dump_1755.bin", std::ios::binary);
    f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)(out.size() * sizeof(float)));
    if (!f) { std::cerr << "cannot write mtt_ev_dump_1755.bin\n"; return 1; }
    std::cout << "Successfully exported mtt_ev_dump_1755.bin\n";
    return 0;
}
