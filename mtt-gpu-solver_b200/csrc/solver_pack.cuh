// solver_pack.cuh — host-side packing of heads-up subgames into the device layout
// of solver_impl.cuh (included by solver.cu only).
#pragma once
#include <thread>
// ====================================================================== host
struct SubPack {
    std::vector<DNode> nodes;
    std::vector<int16_t> depth;      // distance from the root, recomputed from the links
    std::vector<uint8_t> tab;
    std::vector<uint16_t> hcards;
    std::vector<float> range;
    SubDesc d{};
    int status = MTT_OK;
};

static int pad4(int h) { return (h + 3) & ~3; }

static void build_variant(const uint8_t* board, int nboard, int dealt, const int H[2],
                          const std::vector<uint16_t> cards[2], const std::vector<uint16_t> combos[2], uint8_t* out) {
    // hands holding a board card (a card dealt earlier in a flop subgame) or
    // the dealt card are blocked: score 0, no entry positions
    uint64_t bmask = 0;
    for (int k = 0; k < nboard; ++k) bmask |= 1ull << board[k];
    std::vector<uint32_t> sc[2];
    for (int p = 0; p < 2; ++p) {
        sc[p].resize(H[p]);
        for (int h = 0; h < H[p]; ++h) {
            const int c1 = cards[p][h] & 0xFF, c2 = cards[p][h] >> 8;
            if ((dealt >= 0 && (c1 == dealt || c2 == dealt)) || ((bmask >> c1) & 1ull) || ((bmask >> c2) & 1ull)) {
                sc[p][h] = 0u;
                continue;
            }
            Planes pl; planes_clear(pl);
            for (int k = 0; k < nboard; ++k) planes_add(pl, board[k]);
            if (dealt >= 0) planes_add(pl, dealt);
            planes_add(pl, c1);
            planes_add(pl, c2);
            sc[p][h] = score_planes(pl);
        }
    }
    TabView tv = tab_view(out, H[0], H[1]);
    std::vector<uint16_t> sorted[2], cl[2], seg[2];
    std::vector<uint32_t> ssc[2], clsc[2];
    for (int p = 0; p < 2; ++p) {
        sorted[p].resize(H[p]);
        std::iota(sorted[p].begin(), sorted[p].end(), (uint16_t)0);
        std::stable_sort(sorted[p].begin(), sorted[p].end(), [&](uint16_t x, uint16_t y) { return sc[p][x] < sc[p][y]; });
        ssc[p].resize(H[p]);
        for (int i = 0; i < H[p]; ++i) ssc[p][i] = sc[p][sorted[p][i]];
        // per card lists in rank order
        std::vector<std::vector<uint16_t>> by(52);
        for (int i = 0; i < H[p]; ++i) {
            const uint16_t h = sorted[p][i];
            by[cards[p][h] & 0xFF].push_back(h);
            by[cards[p][h] >> 8].push_back(h);
        }
        seg[p].assign(54, 0);
        cl[p].clear();
        for (int c = 0; c < 52; ++c) {
            seg[p][c] = (uint16_t)cl[p].size();
            for (uint16_t h : by[c]) cl[p].push_back(h);
        }
        seg[p][52] = seg[p][53] = (uint16_t)cl[p].size();
        clsc[p].resize(cl[p].size());
        for (size_t e = 0; e < cl[p].size(); ++e) clsc[p][e] = sc[p][cl[p][e]];
        std::memcpy(const_cast<uint16_t*>(tv.sorted[p]), sorted[p].data(), 2 * (size_t)H[p]);
        std::memcpy(const_cast<uint16_t*>(tv.cl[p]), cl[p].data(), 2 * cl[p].size());
        std::memcpy(const_cast<uint16_t*>(tv.seg[p]), seg[p].data(), 2 * 54);
    }
    for (int q = 0; q < 2; ++q) {
        const int o = 1 - q;
        Entry* ent = const_cast<Entry*>(tv.ent[q]);
        for (int h = 0; h < H[q]; ++h) {
            Entry e{};
            const int c1 = cards[q][h] & 0xFF, c2 = cards[q][h] >> 8;
            e.c1 = (uint8_t)c1;
            e.c2 = (uint8_t)c2;
            if ((dealt >= 0 && (c1 == dealt || c2 == dealt)) || ((bmask >> c1) & 1ull) || ((bmask >> c2) & 1ull)) {
                e.lt = e.le = 0xFFFFu;
                e.same = -1;
                ent[h] = e;
                continue;
            }
            const uint32_t s = sc[q][h];
            e.lt = (uint16_t)(std::lower_bound(ssc[o].begin(), ssc[o].end(), s) - ssc[o].begin());
            e.le = (uint16_t)(std::upper_bound(ssc[o].begin(), ssc[o].end(), s) - ssc[o].begin());
            auto seg_pos = [&](int c, bool upper) {
                auto b = clsc[o].begin() + seg[o][c], en = clsc[o].begin() + seg[o][c + 1];
                return (uint8_t)((upper ? std::upper_bound(b, en, s) : std::lower_bound(b, en, s)) - b);
            };
            e.ltc1 = seg_pos(c1, false);
            e.lec1 = seg_pos(c1, true);
            e.ltc2 = seg_pos(c2, false);
            e.lec2 = seg_pos(c2, true);
            const uint16_t cid = combos[q][h];
            auto it = std::lower_bound(combos[o].begin(), combos[o].end(), cid);
            e.same = (it != combos[o].end() && *it == cid) ? (int16_t)(it - combos[o].begin()) : (int16_t)-1;
            ent[h] = e;
        }
    }
}

static void combo_cards(int id, int& c1, int& c2) {
    int a = 0, row = 51, k = id;
    while (k >= row) { k -= row; ++a; --row; }
    c1 = a;
    c2 = a + 1 + k;
}

static void pack_one(const mtt_subgame& g, SubPack& sp) {
    sp.status = MTT_OK;
    int rows[2] = {g.rows[0], g.rows[1]};
    if (!g.nodes || g.n_nodes <= 0 || g.nboard < 3 || g.nboard > 5) { sp.status = MTT_ERR_INVALID; return; }
    int st = validate_tree(g.nodes, g.n_nodes, rows);
    if (st) { sp.status = st; return; }
    uint64_t bm = 0;
    for (int k = 0; k < g.nboard; ++k) {
        if (g.board[k] > 51 || ((bm >> g.board[k]) & 1ull)) { sp.status = MTT_ERR_INVALID; return; }
        bm |= 1ull << g.board[k];
    }
    const int H[2] = {g.H[0], g.H[1]};
    std::vector<uint16_t> combos[2], cards[2];
    for (int p = 0; p < 2; ++p) {
        if (H[p] < 1 || H[p] > 1326 || !g.combos[p] || !g.ranges[p]) { sp.status = MTT_ERR_INVALID; return; }
        combos[p].assign(g.combos[p], g.combos[p] + H[p]);
        cards[p].resize(H[p]);
        for (int h = 0; h < H[p]; ++h) {
            const int id = combos[p][h];
            if (id >= 1326 || (h > 0 && combos[p][h - 1] >= id)) { sp.status = MTT_ERR_INVALID; return; }
            int c1, c2;
            combo_cards(id, c1, c2);
            if (((bm >> c1) & 1ull) || ((bm >> c2) & 1ull)) { sp.status = MTT_ERR_INVALID; return; }
            const float r = g.ranges[p][h];
            if (!(r >= 0.0f) || !std::isfinite(r)) { sp.status = MTT_ERR_INVALID; return; }
            cards[p][h] = (uint16_t)(c1 | (c2 << 8));
        }
    }
    const int nn = g.n_nodes;
    const int Hp[2] = {pad4(H[0]), pad4(H[1])};
    // nodes
    sp.nodes.assign(nn, DNode{});
    std::vector<int> rsrc0(nn, 0), rsrc1(nn, 0), dealt(nn, -1), dealt0(nn, -1);
    std::vector<uint64_t> dm(nn, 0ull);      // cards dealt above (and at) each node
    for (int i = 0; i < nn; ++i) {
        const mtt_node& m = g.nodes[i];
        DNode& d = sp.nodes[i];
        d.type = m.type;
        d.player = m.player;
        d.na = (m.type == MTT_NODE_DECISION || m.type == MTT_NODE_CHANCE) ? m.num_actions : 0;
        d.wmask = m.active_mask;
        d.first = m.children_offset;
        d.row = m.infoset_offset;
        d.pot = m.pot_size;
        d.c0 = m.committed[0];
        d.c1 = m.committed[1];
        if (m.type == MTT_NODE_DECISION && m.num_actions > MAXA) { sp.status = MTT_ERR_UNSUPPORTED; return; }
        if ((m.type == MTT_NODE_CHANCE && g.nboard == 5) || (m.type == MTT_NODE_LEAF && g.nboard != 4)) {
            sp.status = MTT_ERR_INVALID;
            return;
        }
    }
    sp.depth.assign(nn, 0);
    for (int i = 0; i < nn; ++i) {
        const mtt_node& m = g.nodes[i];
        if (m.type == MTT_NODE_DECISION || m.type == MTT_NODE_CHANCE)
            for (int k = 0; k < m.num_actions; ++k) sp.depth[m.children_offset + k] = (int16_t)(sp.depth[i] + 1);
        if (m.type == MTT_NODE_DECISION) {
            for (int k = 0; k < m.num_actions; ++k) {
                const int c = m.children_offset + k;
                rsrc0[c] = m.player == 0 ? c : rsrc0[i];
                rsrc1[c] = m.player == 1 ? c : rsrc1[i];
                dealt[c] = dealt[i];
                dealt0[c] = dealt0[i];
                dm[c] = dm[i];
            }
        } else if (m.type == MTT_NODE_CHANCE) {
            for (int k = 0; k < m.num_actions; ++k) {
                const int c = m.children_offset + k;
                rsrc0[c] = c;
                rsrc1[c] = c;
                dealt[c] = g.nodes[c].turn_idx;
                dealt0[c] = dealt[i];
                if (dealt[c] < 0 || dealt[c] > 51 || (((bm | dm[i]) >> dealt[c]) & 1ull)) {
                    sp.status = MTT_ERR_INVALID;
                    return;
                }
                dm[c] = dm[i] | (1ull << dealt[c]);
            }
            // cards already dealt above a chance node leave no second deal on a 5-card board
            if (g.nboard + __builtin_popcountll(dm[i]) >= 5) { sp.status = MTT_ERR_INVALID; return; }
        }
    }
    for (int i = 0; i < nn; ++i) {
        sp.nodes[i].reach_src0 = rsrc0[i];
        sp.nodes[i].reach_src1 = rsrc1[i];
        sp.nodes[i].dealt = (int16_t)dealt[i];
        sp.nodes[i].dealt0 = (int16_t)dealt0[i];
        sp.nodes[i].nlive = 52 - g.nboard - __builtin_popcountll(dm[i]);
        // variants: 5-card boards one; turn subgames one per dealt card, 52 =
        // none; flop subgames 0 = none, 1 + t = turn card t, 53 + 52 t + r =
        // turn t then river r
        int var = 0;
        if (g.nboard == 4) var = dealt[i] < 0 ? 52 : dealt[i];
        else if (g.nboard == 3) var = dealt[i] < 0 ? 0 : (dealt0[i] < 0 ? 1 + dealt[i] : 53 + 52 * dealt0[i] + dealt[i]);
        sp.nodes[i].var = var;
        // a showdown needs all five board cards
        if (g.nodes[i].type == MTT_NODE_SHOWDOWN && g.nboard + __builtin_popcountll(dm[i]) != 5) {
            sp.status = MTT_ERR_INVALID;
            return;
        }
        // a depth-limit leaf stands for the river deal, so none sits below one
        if (g.nodes[i].type == MTT_NODE_LEAF && dealt[i] >= 0) { sp.status = MTT_ERR_INVALID; return; }
    }
    // tables
    const int vsize = tab_variant_bytes(H[0], H[1]);
    const int nvar = g.nboard == 5 ? 1 : (g.nboard == 4 ? 53 : 53 + 52 * 52);
    sp.tab.assign((size_t)vsize * nvar, 0);
    if (g.nboard == 5) {
        build_variant(g.board, 5, -1, H, cards, combos, sp.tab.data());
    } else if (g.nboard == 3) {
        // the variants some terminal uses, built on host threads
        std::vector<char> used(nvar, 0);
        for (int i = 0; i < nn; ++i)
            if (g.nodes[i].type == MTT_NODE_FOLD || g.nodes[i].type == MTT_NODE_SHOWDOWN) used[sp.nodes[i].var] = 1;
        std::vector<int> todo;
        for (int v = 0; v < nvar; ++v) if (used[v]) todo.push_back(v);
        auto build = [&](int v) {
            uint8_t bd[5] = {g.board[0], g.board[1], g.board[2], 0, 0};
            uint8_t* dst = sp.tab.data() + (size_t)vsize * v;
            if (v == 0) {
                build_variant(bd, 3, -1, H, cards, combos, dst);
            } else if (v < 53) {
                build_variant(bd, 3, v - 1, H, cards, combos, dst);
            } else {
                bd[3] = (uint8_t)((v - 53) / 52);
                build_variant(bd, 4, (v - 53) % 52, H, cards, combos, dst);
            }
        };
        const int nthr = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 16));
        std::vector<std::thread> th;
        for (int t = 0; t < nthr; ++t)
            th.emplace_back([&, t]() { for (size_t k = t; k < todo.size(); k += nthr) build(todo[k]); });
        for (auto& x : th) x.join();
    } else {
        for (int c = 0; c < 52; ++c) {
            if ((bm >> c) & 1ull) continue;
            build_variant(g.board, 4, c, H, cards, combos, sp.tab.data() + (size_t)vsize * c);
        }
        build_variant(g.board, 4, -1, H, cards, combos, sp.tab.data() + (size_t)vsize * 52);
    }
    sp.hcards.assign((size_t)Hp[0] + Hp[1], 0xFFFFu);
    sp.range.assign((size_t)Hp[0] + Hp[1], 0.0f);
    for (int h = 0; h < H[0]; ++h) { sp.hcards[h] = cards[0][h]; sp.range[h] = g.ranges[0][h]; }
    for (int h = 0; h < H[1]; ++h) { sp.hcards[Hp[0] + h] = cards[1][h]; sp.range[Hp[0] + h] = g.ranges[1][h]; }
    SubDesc& d = sp.d;
    d.n_nodes = nn;
    d.H0 = H[0]; d.H1 = H[1];
    d.Hp0 = Hp[0]; d.Hp1 = Hp[1];
    d.rows0 = rows[0]; d.rows1 = rows[1];
    d.tab_vsize = vsize;
    d.n_live = 52 - g.nboard;
    d.river = g.nboard == 5 ? 1 : 0;
    d.var_none = g.nboard == 5 ? 0 : (g.nboard == 4 ? 52 : 0);
    d.pot = g.nodes[0].pot_size;
}

