// tree.cpp — heads-up betting-tree builder and validator (host).
//
// The reference ships no tree builder (its solver mains are stubs,
// honest_multistreet_solver.cu:251-254); its kernels consume a flat array of
// FlatNode (honest_multistreet_solver.cu:16-21) whose children are
// contiguous.  This builder produces that layout breadth-first, so every
// parent precedes its children and a single forward pass over the array is a
// valid top-down order (and the reverse a bottom-up order).
//
// Action order at a decision node: [fold] [check|call] bets/raises by size
// ascending, all-in last.  Sizes at or above the remaining stack collapse into
// all-in; equal amounts are offered once.
#include <algorithm>
#include <cmath>
#include <deque>
#include <vector>

#include "mtt_common.h"

namespace mtt {

struct BState {
    float c[2];        // chips committed, including half of the starting pot each
    float rem[2];      // chips behind; exactly 0 once a player is all-in
    int to_act;
    int raises;        // raises made after the first bet of this street
    bool bet_open;     // a bet is live this street
    bool first_checked;
    int street;        // 3 flop, 4 turn, 5 river
};

struct Pending {
    int idx;
    int kind;          // 0 decision, 1 chance (deal the river), 2 all-in chance (river then showdown)
    BState st;
};

// Amounts within this relative tolerance of the stack are all-in.
constexpr float kAllInTol = 1e-5f;
static bool reaches(float amount, float rem) { return amount >= rem * (1.0f - kAllInTol); }

int build_tree(const mtt_tree_spec& sp, const uint8_t* /*board*/, std::vector<mtt_node>& out,
               int rows[2], int* max_depth) {
    if (!(sp.pot > 0.0f) || sp.stack < 0.0f || sp.n_bet_sizes < 0 || sp.n_bet_sizes > MTT_MAX_SIZES ||
        sp.n_raise_sizes < 0 || sp.n_raise_sizes > MTT_MAX_SIZES || sp.raise_cap < 0 ||
        sp.street < 3 || sp.street > 5 || (sp.river_leaves && sp.street != 4) || (sp.river_runout && sp.street == 5) ||
        (sp.river_leaves && sp.river_runout))
        return MTT_ERR_INVALID;
    for (int i = 0; i < sp.n_bet_sizes; ++i) if (!(sp.bet_sizes[i] > 0.0f)) return MTT_ERR_INVALID;
    for (int i = 0; i < sp.n_raise_sizes; ++i) if (!(sp.raise_sizes[i] > 0.0f)) return MTT_ERR_INVALID;
    const float* rsz = sp.n_raise_sizes > 0 ? sp.raise_sizes : sp.bet_sizes;
    const int nrs = sp.n_raise_sizes > 0 ? sp.n_raise_sizes : sp.n_bet_sizes;

    out.clear();
    rows[0] = rows[1] = 0;
    int maxd = 0;
    std::deque<Pending> q;
    auto make_node = [&](int depth) {
        mtt_node n{};
        n.turn_idx = -1;
        n.depth = (int16_t)depth;
        out.push_back(n);
        return (int)out.size() - 1;
    };
    BState root{};
    root.c[0] = root.c[1] = 0.5f * sp.pot;
    root.rem[0] = root.rem[1] = sp.stack;
    root.to_act = 0;
    root.street = sp.street;
    int r = make_node(0);
    q.push_back({r, 0, root});
    const int kMaxNodes = 1 << 24;

    while (!q.empty()) {
        Pending pd = q.front();
        q.pop_front();
        const int me = pd.idx;
        const int depth = out[me].depth;
        if (depth > maxd) maxd = depth;
        BState s = pd.st;
        if ((int)out.size() > kMaxNodes) return MTT_ERR_UNSUPPORTED;
        out[me].pot_size = s.c[0] + s.c[1];
        out[me].committed[0] = s.c[0];
        out[me].committed[1] = s.c[1];

        if (pd.kind == 1 || pd.kind == 2) {   // river chance node (turn trees only)
            out[me].type = MTT_NODE_CHANCE;
            out[me].player = 0;
            const int first = (int)out.size();
            // children: every card not on the 4-card board, ascending; the
            // board cards are unknown here, so all 52 are listed and the
            // caller's board removes 4 (see mtt_tree_build_for_board).
            out[me].children_offset = first;
            out[me].num_actions = 0;
            out[me].reserved = std::min(s.rem[0], s.rem[1]);   // chips behind at the deal
            (void)first;
            continue;   // finished by the board-aware wrapper
        }

        const int p = s.to_act, o = 1 - p;
        out[me].type = MTT_NODE_DECISION;
        out[me].player = (uint8_t)p;
        const float to_call = s.c[o] - s.c[p];
        const float rem_p = s.rem[p], rem_o = s.rem[o];
        const float pot = s.c[0] + s.c[1];

        struct Act { int type; float amount; };   // 0 fold, 1 check/call, 2 bet/raise (amount added)
        std::vector<Act> acts;
        if (to_call > 0.0f) {
            acts.push_back({0, 0.0f});
            acts.push_back({1, to_call});
            if (s.raises < sp.raise_cap && !reaches(to_call, rem_p) && rem_o > 0.0f) {
                std::vector<float> amts;
                for (int i = 0; i < nrs; ++i) {
                    float a = to_call + rsz[i] * (pot + to_call);
                    if (reaches(a, rem_p)) a = rem_p;
                    amts.push_back(a);
                }
                if (sp.allin) amts.push_back(rem_p);
                std::sort(amts.begin(), amts.end());
                amts.erase(std::unique(amts.begin(), amts.end()), amts.end());
                for (float a : amts) acts.push_back({2, a});
            }
        } else {
            acts.push_back({1, 0.0f});
            if (rem_p > 0.0f) {
                std::vector<float> amts;
                for (int i = 0; i < sp.n_bet_sizes; ++i) {
                    float a = sp.bet_sizes[i] * pot;
                    if (reaches(a, rem_p)) a = rem_p;
                    amts.push_back(a);
                }
                if (sp.allin) amts.push_back(rem_p);
                std::sort(amts.begin(), amts.end());
                amts.erase(std::unique(amts.begin(), amts.end()), amts.end());
                for (float a : amts) acts.push_back({2, a});
            }
        }
        if (acts.size() > 255) return MTT_ERR_UNSUPPORTED;
        out[me].num_actions = (uint8_t)acts.size();
        out[me].infoset_offset = rows[p];
        rows[p] += (int)acts.size();
        const int first = (int)out.size();
        out[me].children_offset = first;
        for (size_t a = 0; a < acts.size(); ++a) make_node(depth + 1);
        for (size_t a = 0; a < acts.size(); ++a) {
            const int ch = first + (int)a;
            BState ns = s;
            const Act& ac = acts[a];
            if (ac.type == 0) {   // fold: the opponent keeps the pot
                mtt_node& cn = out[ch];
                cn.type = MTT_NODE_FOLD;
                cn.player = (uint8_t)p;
                cn.active_mask = (uint8_t)(1u << o);
                cn.pot_size = s.c[0] + s.c[1];
                cn.committed[0] = s.c[0];
                cn.committed[1] = s.c[1];
                if (cn.depth > maxd) maxd = cn.depth;
                continue;
            }
            bool closes = false;
            if (ac.type == 1) {
                if (to_call > 0.0f) {                         // call: match exactly
                    ns.c[p] = s.c[o];
                    ns.rem[p] = reaches(to_call, rem_p) ? 0.0f : rem_p - to_call;
                    closes = true;
                }
                else if (p == 1) closes = true;               // check behind
                else { ns.first_checked = true; ns.to_act = o; }
            } else {
                ns.c[p] += ac.amount;
                ns.rem[p] = (ac.amount == rem_p) ? 0.0f : rem_p - ac.amount;
                if (s.bet_open) ns.raises += 1;
                ns.bet_open = true;
                ns.to_act = o;
            }
            if (!closes) { q.push_back({ch, 0, ns}); continue; }
            const bool all_in = ns.rem[0] <= 0.0f || ns.rem[1] <= 0.0f;
            if (ns.street == 5) {
                mtt_node& cn = out[ch];
                cn.type = MTT_NODE_SHOWDOWN;
                cn.active_mask = 3;
                cn.pot_size = ns.c[0] + ns.c[1];
                cn.committed[0] = ns.c[0];
                cn.committed[1] = ns.c[1];
                if (cn.depth > maxd) maxd = cn.depth;
            } else if (!all_in && sp.river_leaves) {
                mtt_node& cn = out[ch];
                cn.type = MTT_NODE_LEAF;
                cn.pot_size = ns.c[0] + ns.c[1];
                cn.committed[0] = ns.c[0];
                cn.committed[1] = ns.c[1];
                cn.reserved = std::min(ns.rem[0], ns.rem[1]);   // chips behind at the river
                if (cn.depth > maxd) maxd = cn.depth;
            } else {
                BState rs = ns;
                rs.street = 5;
                rs.to_act = 0;
                rs.raises = 0;
                rs.bet_open = false;
                rs.first_checked = false;
                q.push_back({ch, all_in ? 2 : 1, rs});
            }
        }
    }
    *max_depth = maxd;
    return MTT_OK;
}

// Board-aware wrapper.  Turn trees (street 4, 4-card board) and flop trees
// (street 3, 3-card board): every chance node gets one child per card not on
// the board and not dealt above it.  Each child is followed by the next
// street's betting round, grafted from a template built at the chance node's
// commitments, or by showdowns when a player is all-in or the river is a
// runout.  Flop trees always run the river out (flop and turn betting, then
// the river dealt to showdowns, as the reference's multistreet solver);
// turn trees do so with river_runout.  Subtrees are appended breadth-first
// per chance node, keeping children contiguous and after their parent.
int build_tree_board(const mtt_tree_spec& sp, const uint8_t* board, int nboard, std::vector<mtt_node>& out,
                     int rows[2], int* max_depth) {
    if (sp.street == 5) {
        if (nboard != 5 && nboard != 0) return MTT_ERR_INVALID;
        return build_tree(sp, board, out, rows, max_depth);
    }
    if (nboard != sp.street) return MTT_ERR_INVALID;
    int trows[2], tdepth = 0;
    MTT_TRY(build_tree(sp, board, out, trows, &tdepth));
    uint64_t bm = 0;
    for (int k = 0; k < nboard; ++k) {
        if (board[k] > 51 || ((bm >> board[k]) & 1ull)) return MTT_ERR_INVALID;
        bm |= 1ull << board[k];
    }
    rows[0] = trows[0];
    rows[1] = trows[1];
    int maxd = tdepth;
    std::vector<uint64_t> above(out.size(), 0ull);   // cards dealt above each node
    // BFS over chance nodes in index order; appending keeps parents first.
    for (size_t i = 0; i < out.size(); ++i) {
        if (out[i].type != MTT_NODE_CHANCE) continue;
        const uint64_t dm = above[i];
        const int next = sp.street + __builtin_popcountll(dm) + 1;   // street of the round after this deal
        const float c0 = out[i].committed[0], c1 = out[i].committed[1];
        const int cdepth = out[i].depth;
        const float behind = out[i].reserved;
        out[i].reserved = 0.0f;
        const bool all_in = behind <= 0.0f;
        const bool runout = next == 5 && (sp.street == 3 || sp.river_runout);
        std::vector<int> cards;
        for (int c = 0; c < 52; ++c) if (!(((bm | dm) >> c) & 1ull)) cards.push_back(c);
        const int first = (int)out.size();
        out[i].children_offset = first;
        out[i].num_actions = (uint8_t)cards.size();
        for (size_t k = 0; k < cards.size(); ++k) {
            mtt_node n{};
            n.turn_idx = (int16_t)cards[k];
            n.depth = (int16_t)(cdepth + 1);
            out.push_back(n);
            above.push_back(dm | (1ull << cards[k]));
        }
        // the next round from this state (none for showdowns or a further deal)
        std::vector<mtt_node> rt;
        int rrows[2] = {0, 0}, rdepth = 0;
        const bool showdowns = next == 5 && (all_in || runout);
        if (!showdowns && !all_in) {
            mtt_tree_spec rs = sp;
            rs.street = next;
            rs.river_leaves = 0;
            rs.river_runout = runout || sp.street == 3;
            // the round starts from the chance node's commitments: express
            // them through a pot/stack pair with the same remaining stacks
            rs.pot = c0 + c1;
            rs.stack = behind;
            MTT_TRY(build_tree(rs, nullptr, rt, rrows, &rdepth));
        }
        for (size_t k = 0; k < cards.size(); ++k) {
            const int ch = first + (int)k;
            if (showdowns || all_in) {
                // all-in before the river: a further deal; else showdowns
                out[ch].type = showdowns ? MTT_NODE_SHOWDOWN : MTT_NODE_CHANCE;
                out[ch].active_mask = showdowns ? 3 : 0;
                out[ch].pot_size = c0 + c1;
                out[ch].committed[0] = c0;
                out[ch].committed[1] = c1;
                out[ch].reserved = 0.0f;
                maxd = std::max(maxd, (int)out[ch].depth);
                continue;
            }
            // graft rt with root at ch: rt[0] -> ch, rt[j>0] appended
            const int base = (int)out.size() - 1;   // rt index j>0 maps to base + j
            for (size_t j = 0; j < rt.size(); ++j) {
                mtt_node n = rt[j];
                if (n.type == MTT_NODE_DECISION) {
                    n.children_offset = base + n.children_offset;
                    n.infoset_offset += rows[n.player];
                }
                n.depth = (int16_t)(rt[j].depth + cdepth + 1);
                n.turn_idx = (int16_t)(j == 0 ? cards[k] : -1);
                maxd = std::max(maxd, (int)n.depth);
                if (j == 0) out[ch] = n;
                else { out.push_back(n); above.push_back(above[ch]); }
            }
            rows[0] += rrows[0];
            rows[1] += rrows[1];
        }
    }
    // commitments inside grafted rounds were expressed relative to rs.pot/2;
    // the builder put c = rs.pot/2 + bets for BOTH players, which equals the
    // true commitments only when c0 == c1 at the chance node (always true:
    // a round closes with equal commitments).
    *max_depth = maxd;
    return MTT_OK;
}

int validate_tree(const mtt_node* nodes, int n, const int rows[2]) {
    if (!nodes || n <= 0) return MTT_ERR_INVALID;
    std::vector<int> parent(n, -1);
    for (int i = 0; i < n; ++i) {
        const mtt_node& nd = nodes[i];
        if (nd.type > MTT_NODE_LEAF) return MTT_ERR_INVALID;
        if (nd.type == MTT_NODE_DECISION || nd.type == MTT_NODE_CHANCE) {
            if (nd.num_actions < 1) return MTT_ERR_INVALID;
            if (nd.children_offset <= i || nd.children_offset + nd.num_actions > n) return MTT_ERR_INVALID;
            for (int a = 0; a < nd.num_actions; ++a) {
                int c = nd.children_offset + a;
                if (parent[c] != -1) return MTT_ERR_INVALID;
                parent[c] = i;
            }
        }
        if (nd.type == MTT_NODE_DECISION) {
            if (nd.player > 1) return MTT_ERR_INVALID;
            if (nd.num_actions > 16) return MTT_ERR_UNSUPPORTED;
            if (nd.infoset_offset < 0 || nd.infoset_offset + nd.num_actions > rows[nd.player])
                return MTT_ERR_INVALID;
        }
        if (nd.type == MTT_NODE_FOLD && nd.active_mask != 1 && nd.active_mask != 2) return MTT_ERR_INVALID;
        if (!(nd.pot_size >= 0.0f) || !std::isfinite(nd.committed[0]) || !std::isfinite(nd.committed[1]))
            return MTT_ERR_INVALID;
    }
    for (int i = 1; i < n; ++i) {
        if (parent[i] < 0) return MTT_ERR_INVALID;   // unreachable node
        if (nodes[parent[i]].type == MTT_NODE_CHANCE && (nodes[i].turn_idx < 0 || nodes[i].turn_idx > 51))
            return MTT_ERR_INVALID;
    }
    return MTT_OK;
}

}  // namespace mtt

extern "C" int mtt_tree_build(const mtt_tree_spec* spec, mtt_node* nodes, int32_t capacity, int32_t* n_nodes,
                              int32_t rows[2], int32_t* max_depth) {
    if (!spec || !n_nodes || !rows || !max_depth) return MTT_ERR_INVALID;
    if (spec->street != 5) return MTT_ERR_INVALID;   // turn trees need the board: mtt_tree_build_board
    std::vector<mtt_node> v;
    int r[2], d = 0;
    MTT_TRY(mtt::build_tree(*spec, nullptr, v, r, &d));
    *n_nodes = (int32_t)v.size();
    rows[0] = r[0];
    rows[1] = r[1];
    *max_depth = d;
    if (nodes) {
        if (capacity < (int32_t)v.size()) return MTT_ERR_INVALID;
        std::copy(v.begin(), v.end(), nodes);
    }
    return MTT_OK;
}

extern "C" int mtt_tree_build_board(const mtt_tree_spec* spec, const uint8_t* board, int32_t nboard,
                                    mtt_node* nodes, int32_t capacity, int32_t* n_nodes, int32_t rows[2],
                                    int32_t* max_depth) {
    if (!spec || !n_nodes || !rows || !max_depth || (nboard > 0 && !board)) return MTT_ERR_INVALID;
    std::vector<mtt_node> v;
    int r[2], d = 0;
    MTT_TRY(mtt::build_tree_board(*spec, board, nboard, v, r, &d));
    *n_nodes = (int32_t)v.size();
    rows[0] = r[0];
    rows[1] = r[1];
    *max_depth = d;
    if (nodes) {
        if (capacity < (int32_t)v.size()) return MTT_ERR_INVALID;
        std::copy(v.begin(), v.end(), nodes);
    }
    return MTT_OK;
}

extern "C" int mtt_tree_validate(const mtt_node* nodes, int32_t n_nodes, int32_t rows[2]) {
    if (!rows) return MTT_ERR_INVALID;
    int r[2] = {rows[0], rows[1]};
    return mtt::validate_tree(nodes, n_nodes, r);
}
