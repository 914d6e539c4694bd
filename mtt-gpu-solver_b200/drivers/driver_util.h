// driver_util.h — shared helpers of the command-line drivers (host only):
// status checks, card parsing, combos and seeded Dirichlet ranges.
#pragma once
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mtt_b200.h"

#define DRV_CHECK(call)                                                                          \
    do {                                                                                         \
        const int s_ = (call);                                                                   \
        if (s_ != MTT_OK) {                                                                      \
            std::fprintf(stderr, "%s failed: status %d (cuda %d)\n", #call, s_, mtt_last_cuda_error()); \
            std::exit(1);                                                                        \
        }                                                                                        \
    } while (0)
#define DRV_CUDA(call)                                                                           \
    do {                                                                                         \
        const cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                                 \
            std::fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));              \
            std::exit(1);                                                                        \
        }                                                                                        \
    } while (0)

// "AsKd7c" or "51,46,23": cards rank*4 + suit, rank 0 = '2' .. 12 = 'A', suits c d h s.
inline std::vector<int> parse_cards(const std::string& s) {
    std::vector<int> out;
    if (s.find(',') != std::string::npos || (s.size() && std::isdigit((unsigned char)s[0]))) {
        size_t p = 0;
        while (p < s.size()) {
            size_t q = s.find(',', p);
            out.push_back(std::atoi(s.substr(p, q == std::string::npos ? std::string::npos : q - p).c_str()));
            if (q == std::string::npos) break;
            p = q + 1;
        }
        return out;
    }
    const std::string ranks = "23456789TJQKA", suits = "cdhs";
    for (size_t i = 0; i + 1 < s.size(); i += 2) {
        const size_t r = ranks.find((char)std::toupper((unsigned char)s[i])), u = suits.find((char)std::tolower((unsigned char)s[i + 1]));
        if (r == std::string::npos || u == std::string::npos) return {};
        out.push_back((int)(r * 4 + u));
    }
    return out;
}

// Lexicographic combo ids (a < b) of the 1,326 pairs that avoid the board.
inline std::vector<uint16_t> live_combos(const std::vector<int>& board) {
    uint64_t bm = 0;
    for (int c : board) bm |= 1ull << c;
    std::vector<uint16_t> out;
    int id = 0;
    for (int a = 0; a < 52; ++a)
        for (int b = a + 1; b < 52; ++b, ++id)
            if (!(((bm >> a) | (bm >> b)) & 1ull)) out.push_back((uint16_t)id);
    return out;
}

// Dirichlet(alpha) weights over n entries (alpha <= 0: uniform), summing to 1.
inline std::vector<float> dirichlet(std::mt19937_64& rng, size_t n, double alpha) {
    std::vector<double> w(n, 1.0);
    if (alpha > 0.0) {
        std::gamma_distribution<double> g(alpha, 1.0);
        for (auto& x : w) x = g(rng);
    }
    double s = 0.0;
    for (double x : w) s += x;
    std::vector<float> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = (float)(w[i] / s);
    return out;
}

// k distinct cards from 52 not in `used`.
inline std::vector<int> draw_cards(std::mt19937_64& rng, int k, uint64_t used = 0) {
    std::vector<int> out;
    std::uniform_int_distribution<int> d(0, 51);
    while ((int)out.size() < k) {
        const int c = d(rng);
        if ((used >> c) & 1ull) continue;
        used |= 1ull << c;
        out.push_back(c);
    }
    return out;
}

inline std::vector<float> parse_floats(const std::string& s) {
    std::vector<float> out;
    size_t p = 0;
    while (p < s.size()) {
        size_t q = s.find(',', p);
        out.push_back((float)std::atof(s.substr(p, q == std::string::npos ? std::string::npos : q - p).c_str()));
        if (q == std::string::npos) break;
        p = q + 1;
    }
    return out;
}
