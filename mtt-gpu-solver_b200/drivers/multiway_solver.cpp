// multiway_solver — four-player ICM river driver.  The reference builds an
// executable of this name whose main only prints a line
// (src/postflop/multiway_4way_engine.cu:259-262); this one runs its engine
// (multiway_4way_engine.cu:41-257) on a seeded spot:  eight seats with stacks
// lognormal(log 20 bb, 0.5), seats 0-3 in the hand with Malmuth-Harville
// bubble factors for payouts 50/30/20, a seeded river board, Dirichlet(0.3)
// ranges over the live combos, bets {50%, 100%} and one pot-sized raise over
// --pot bb of dead money, CFR+ with simultaneous updates as the reference.
#include <chrono>
#include <cmath>
#include <iomanip>
#include <iostream>

#include "driver_util.h"

int main(int argc, char** argv) {
    int iters = 200, seed = 4, semantics = MTT_SEM_CORRECT;
    double pot = 4.0, alpha = 0.3;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() { return std::string(i + 1 < argc ? argv[++i] : ""); };
        if (a == "--iters") iters = std::atoi(val().c_str());
        else if (a == "--seed") seed = std::atoi(val().c_str());
        else if (a == "--pot") pot = std::atof(val().c_str());
        else if (a == "--range-alpha") alpha = std::atof(val().c_str());
        else if (a == "--semantics") semantics = val() == "reference" ? MTT_SEM_REFERENCE : MTT_SEM_CORRECT;
        else {
            std::cout << "usage: multiway_solver [--iters 200] [--seed N] [--pot 4] [--range-alpha 0.3]"
                         " [--semantics correct|reference]\n";
            return a == "--help" || a == "-h" ? 0 : 1;
        }
    }
    std::mt19937_64 rng((uint64_t)seed * 0x9E3779B97F4A7C15ull + 11);
    std::lognormal_distribution<double> ln(std::log(20.0), 0.5);
    std::vector<double> stacks(8);
    for (auto& s : stacks) s = ln(rng);
    const double payouts[3] = {0.5, 0.3, 0.2};
    const int32_t seats[4] = {0, 1, 2, 3};
    double bf[16];
    DRV_CHECK(mtt_icm_bubble_factors(stacks.data(), 8, payouts, 3, seats, 4, bf));
    const std::vector<int> board = draw_cards(rng, 5);
    const std::vector<uint16_t> combos = live_combos(board);
    std::vector<std::vector<float>> ranges(4);
    for (auto& r : ranges) r = dirichlet(rng, combos.size(), alpha);
    mtt_mw_spec sp{};
    sp.pot = (float)pot;
    for (int p = 0; p < 4; ++p) sp.stacks[p] = (float)(stacks[p] - pot / 4.0);
    sp.n_bet_sizes = 2;
    sp.bet_sizes[0] = 0.5f;
    sp.bet_sizes[1] = 1.0f;
    sp.raise_size = 1.0f;
    sp.raise_cap = 1;
    int32_t nn = 0, rows[4], depth = 0;
    DRV_CHECK(mtt_mw_tree_build(&sp, nullptr, 0, &nn, rows, &depth));
    std::vector<mtt_mw_node> nodes(nn);
    DRV_CHECK(mtt_mw_tree_build(&sp, nodes.data(), nn, &nn, rows, &depth));
    mtt_mw_subgame g{};
    g.nodes = nodes.data();
    g.n_nodes = nn;
    for (int p = 0; p < 4; ++p) { g.rows[p] = rows[p]; g.ranges[p] = ranges[p].data(); }
    for (int k = 0; k < 5; ++k) g.board[k] = (uint8_t)board[k];
    g.H = (int32_t)combos.size();
    g.combos = combos.data();
    for (int k = 0; k < 16; ++k) g.bubble[k] = (float)bf[k];
    const auto t0 = std::chrono::steady_clock::now();
    mtt_mw_batch* b = nullptr;
    DRV_CHECK(mtt_mw_batch_create(&g, 1, &b));
    mtt_solve_params p{};
    p.iters = iters; p.algo = MTT_ALGO_CFRPLUS; p.semantics = semantics; p.avg_power = 1.0f;
    DRV_CHECK(mtt_mw_batch_solve(b, &p, 1, nullptr));
    double ev[4];
    DRV_CHECK(mtt_mw_batch_values(b, ev, nullptr));
    const auto t1 = std::chrono::steady_clock::now();
    mtt_mw_batch_destroy(b);
    std::cout << "4-player river: " << nn << " nodes, " << combos.size() << " combos, " << iters << " CFR+ iterations ("
              << (semantics == MTT_SEM_REFERENCE ? "reference" : "correct") << " semantics)\n" << std::fixed;
    for (int q = 0; q < 4; ++q)
        std::cout << "player " << q << ": stack " << std::setprecision(2) << stacks[q] << " bb, bubble factor "
                  << std::setprecision(3) << bf[q * 4 + q] << ", EV " << std::setprecision(6) << ev[q] << " bb\n";
    std::cout << "solve " << std::setprecision(1) << std::chrono::duration<double, std::milli>(t1 - t0).count()
              << " ms\n";
    return 0;
}
