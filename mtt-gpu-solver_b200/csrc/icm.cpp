// icm.cpp — Malmuth-Harville tournament equity and bubble factors (FP64, host).
//
// The probability that the players in set A take the first |A| places, in
// any order, obeys g(A) = sum_{j in A} g(A \ j) * s_j / (S - s(A \ j)) with
// g({}) = 1 (Malmuth-Harville: each next place goes to a remaining player
// with probability proportional to its stack).  Seat i then takes place
// |A| + 1 with probability g(A) * s_i / (S - s(A)) for every A not holding i,
// so equity_i = sum_A g(A) * s_i / (S - s(A)) * payouts[|A|], over |A| < m.
// One pass over the 2^n subsets, O(2^n n).
#include <cmath>
#include <vector>

#include "mtt_common.h"

namespace {
constexpr int kMaxSeats = 16;

int icm_equity(const double* stacks, int n, const double* payouts, int m, double* out) {
    if (!stacks || !payouts || !out || n < 1 || n > kMaxSeats || m < 0 || m > n) return MTT_ERR_INVALID;
    double S = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!(stacks[i] >= 0.0) || !std::isfinite(stacks[i])) return MTT_ERR_INVALID;
        S += stacks[i];
    }
    for (int i = 0; i < n; ++i) out[i] = 0.0;
    if (!(S > 0.0)) return MTT_ERR_INVALID;
    const unsigned full = 1u << n;
    std::vector<double> g(full, 0.0), sA(full, 0.0);
    g[0] = 1.0;
    for (unsigned A = 1; A < full; ++A) {
        const int low = __builtin_ctz(A);
        sA[A] = sA[A & (A - 1)] + stacks[low];
    }
    for (unsigned A = 0; A < full; ++A) {
        const int k = __builtin_popcount(A);
        if (k >= m || g[A] == 0.0) continue;
        const double rest = S - sA[A];
        if (!(rest > 0.0)) continue;
        for (int i = 0; i < n; ++i) {
            if ((A >> i) & 1u) continue;
            const double p = g[A] * stacks[i] / rest;
            out[i] += p * payouts[k];
            g[A | (1u << i)] += p;   // A | i has k + 1 members: visited after A
        }
    }
    return MTT_OK;
}
}  // namespace

extern "C" int mtt_icm_equity(const double* stacks, int32_t n, const double* payouts, int32_t m, double* out) {
    return icm_equity(stacks, n, payouts, m, out);
}

extern "C" int mtt_icm_bubble_factors(const double* stacks, int32_t n, const double* payouts, int32_t m,
                                      const int32_t* seats, int32_t np, double* bf) {
    if (!stacks || !seats || !bf || np < 1 || np > 4 || n < 1 || n > kMaxSeats) return MTT_ERR_INVALID;
    for (int k = 0; k < np; ++k) {
        if (seats[k] < 0 || seats[k] >= n) return MTT_ERR_INVALID;
        for (int j = 0; j < k; ++j) if (seats[j] == seats[k]) return MTT_ERR_INVALID;
    }
    std::vector<double> now(n), win(n), lose(n), st(stacks, stacks + n);
    MTT_TRY(icm_equity(stacks, n, payouts, m, now.data()));
    for (int k = 0; k < np; ++k) {
        double field = 0.0;
        int cnt = 0;
        for (int j = 0; j < np; ++j) {
            if (j == k) continue;
            const int a = seats[k], c = seats[j];
            const double X = std::fmin(stacks[a], stacks[c]);
            double f = 1.0;
            if (X > 0.0) {
                st[a] = stacks[a] + X; st[c] = stacks[c] - X;
                MTT_TRY(icm_equity(st.data(), n, payouts, m, win.data()));
                st[a] = stacks[a] - X; st[c] = stacks[c] + X;
                MTT_TRY(icm_equity(st.data(), n, payouts, m, lose.data()));
                st[a] = stacks[a]; st[c] = stacks[c];
                const double gain = win[a] - now[a], loss = now[a] - lose[a];
                f = gain > 0.0 ? loss / gain : 1.0;
            }
            bf[k * np + j] = f;
            field += f;
            ++cnt;
        }
        bf[k * np + k] = cnt ? field / cnt : 1.0;
    }
    return MTT_OK;
}
