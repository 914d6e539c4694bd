// hu_solver — heads-up CFR+/DCFR solver driver.  The reference builds an
// executable of this name whose main only prints a line
// (src/postflop/honest_multistreet_solver.cu:251-254); this one runs its
// sweeps (honest_multistreet_solver.cu:88-249, batched and scan-based) on a
// tree from the flags and prints the root values and the FP64 exploitability.
//   --config 0: river, uniform 1,081-combo ranges, pot 100, stack 200,
//               bets 50/100% + all-in, 1 raise, 1,000 alternating CFR+ iterations;
//   --config 1: turn + river, Dirichlet(0.3) ranges, pot 60, stack 470,
//               bets 33/75/150% + all-in, 2 raises, DCFR(1.5, 0, 2) x 500;
//   --street 3: a flop subgame (turn chance layer, river run out).
#include <chrono>
#include <iomanip>
#include <iostream>

#include "driver_util.h"

int main(int argc, char** argv) {
    int config = 0, street = -1, iters = -1, raise_cap = -1, seed = 0, semantics = MTT_SEM_CORRECT, algo = -1;
    int alternate = 1, allin = 1;
    float pot = -1.0f, stack = -1.0f, alpha = 1.5f, beta = 0.0f, gamma = 2.0f;
    double range_alpha = -1.0;
    std::string board_s, bets_s;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() { return std::string(i + 1 < argc ? argv[++i] : ""); };
        if (a == "--config") config = std::atoi(val().c_str());
        else if (a == "--board") board_s = val();
        else if (a == "--street") street = std::atoi(val().c_str());
        else if (a == "--pot") pot = (float)std::atof(val().c_str());
        else if (a == "--stack") stack = (float)std::atof(val().c_str());
        else if (a == "--bets") bets_s = val();
        else if (a == "--raise-cap") raise_cap = std::atoi(val().c_str());
        else if (a == "--no-allin") allin = 0;
        else if (a == "--iters") iters = std::atoi(val().c_str());
        else if (a == "--algo") algo = val() == "dcfr" ? MTT_ALGO_DCFR : MTT_ALGO_CFRPLUS;
        else if (a == "--alpha") alpha = (float)std::atof(val().c_str());
        else if (a == "--beta") beta = (float)std::atof(val().c_str());
        else if (a == "--gamma") gamma = (float)std::atof(val().c_str());
        else if (a == "--semantics") semantics = val() == "reference" ? MTT_SEM_REFERENCE : MTT_SEM_CORRECT;
        else if (a == "--simultaneous") alternate = 0;
        else if (a == "--range-alpha") range_alpha = std::atof(val().c_str());
        else if (a == "--seed") seed = std::atoi(val().c_str());
        else {
            std::cout << "usage: hu_solver [--config 0|1] [--street 5|4|3] [--board AsKd7c2h3s] [--pot P] [--stack S]\n"
                         "                 [--bets 0.5,1.0] [--raise-cap N] [--no-allin] [--iters N] [--algo cfrplus|dcfr]\n"
                         "                 [--alpha A --beta B --gamma G] [--semantics correct|reference] [--simultaneous]\n"
                         "                 [--range-alpha 0 (uniform) | a (Dirichlet)] [--seed N]\n";
            return a == "--help" || a == "-h" ? 0 : 1;
        }
    }
    // the configuration's values, then the flags over them
    const bool turn = config == 1;
    if (street < 0) street = turn ? 4 : 5;
    if (pot < 0) pot = turn ? 60.0f : 100.0f;
    if (stack < 0) stack = turn ? 470.0f : 200.0f;
    if (raise_cap < 0) raise_cap = turn ? 2 : 1;
    if (iters < 0) iters = turn ? 500 : 1000;
    if (algo < 0) algo = turn ? MTT_ALGO_DCFR : MTT_ALGO_CFRPLUS;
    if (range_alpha < 0) range_alpha = turn ? 0.3 : 0.0;
    std::vector<float> bets = bets_s.empty() ? (turn ? std::vector<float>{0.33f, 0.75f, 1.5f} : std::vector<float>{0.5f, 1.0f})
                                             : parse_floats(bets_s);
    std::mt19937_64 rng((uint64_t)seed * 0x9E3779B97F4A7C15ull + 7);
    std::vector<int> board = board_s.empty() ? draw_cards(rng, street) : parse_cards(board_s);
    if ((int)board.size() != street || bets.empty() || bets.size() > MTT_MAX_SIZES) {
        std::cerr << "the board must have " << street << " cards and 1-" << MTT_MAX_SIZES << " bet sizes\n";
        return 1;
    }
    mtt_tree_spec sp{};
    sp.pot = pot;
    sp.stack = stack;
    sp.n_bet_sizes = (int32_t)bets.size();
    for (size_t k = 0; k < bets.size(); ++k) sp.bet_sizes[k] = bets[k];
    sp.raise_cap = raise_cap;
    sp.allin = allin;
    sp.street = street;
    std::vector<uint8_t> bd(board.begin(), board.end());
    int32_t nn = 0, rows[2], depth = 0;
    DRV_CHECK(mtt_tree_build_board(&sp, bd.data(), (int32_t)bd.size(), nullptr, 0, &nn, rows, &depth));
    std::vector<mtt_node> nodes(nn);
    DRV_CHECK(mtt_tree_build_board(&sp, bd.data(), (int32_t)bd.size(), nodes.data(), nn, &nn, rows, &depth));
    const std::vector<uint16_t> combos = live_combos(board);
    std::vector<float> r0 = dirichlet(rng, combos.size(), range_alpha), r1 = dirichlet(rng, combos.size(), range_alpha);
    mtt_subgame g{};
    g.nodes = nodes.data();
    g.n_nodes = nn;
    g.rows[0] = rows[0];
    g.rows[1] = rows[1];
    for (size_t k = 0; k < bd.size(); ++k) g.board[k] = bd[k];
    g.nboard = (int32_t)bd.size();
    g.H[0] = g.H[1] = (int32_t)combos.size();
    g.combos[0] = g.combos[1] = combos.data();
    g.ranges[0] = r0.data();
    g.ranges[1] = r1.data();
    const auto t0 = std::chrono::steady_clock::now();
    mtt_batch* b = nullptr;
    DRV_CHECK(mtt_batch_create(&g, 1, &b));
    mtt_solve_params p{};
    p.iters = iters; p.algo = algo; p.alpha = alpha; p.beta = beta; p.gamma = gamma; p.semantics = semantics;
    p.exploitability = 1; p.alternate = alternate; p.avg_power = 2.0f;
    const auto t1 = std::chrono::steady_clock::now();
    DRV_CHECK(mtt_batch_solve_graph(b, &p, nullptr));
    double res[6];
    DRV_CHECK(mtt_batch_results(b, res, nullptr));
    const auto t2 = std::chrono::steady_clock::now();
    mtt_batch_destroy(b);
    static const char* R = "23456789TJQKA";
    static const char* U = "cdhs";
    std::cout << "board ";
    for (int c : board) std::cout << R[c / 4] << U[c % 4];
    std::cout << "  nodes " << nn << "  combos " << combos.size() << "  pot " << pot << "  stack " << stack << "\n"
              << (algo == MTT_ALGO_DCFR ? "DCFR" : "CFR+") << " x " << iters << (alternate ? " (alternating)" : " (simultaneous)")
              << ", " << (semantics == MTT_SEM_REFERENCE ? "reference" : "correct") << " semantics\n"
              << std::fixed << std::setprecision(6)
              << "EV0 " << res[2] << "  EV1 " << res[3] << "  BR0 " << res[0] << "  BR1 " << res[1] << "\n"
              << "exploitability " << std::setprecision(4) << res[5] * 100.0 << " % pot\n"
              << "pack + upload " << std::setprecision(1) << std::chrono::duration<double, std::milli>(t1 - t0).count()
              << " ms, solve " << std::chrono::duration<double, std::milli>(t2 - t1).count() << " ms\n";
    return 0;
}
