// solver_impl.cuh — device-side layout and sweeps of the heads-up CFR solver.
//
// Layout in HBM (all offsets are per subgame, relative to that subgame's base):
//  * DNode[n_nodes] (48 B): the reference FlatNode (honest_multistreet_solver.cu:16-21)
//    plus where each player's reach vector lives and the dealt card.
//  * vectors: every node owns a slot of HS = Hp0 + Hp1 floats in the REACH
//    region and one in the CFV region; player p's part starts at off_p
//    (0 or Hp0).  A decision node writes only its acting player's part of each
//    child's reach slot; the other player's reach is read from the ancestor
//    that last wrote it (reach_src), so it is never copied.  Children are
//    contiguous nodes, so child a's slot is (first + a) * HS.
//  * R_p, S_p: [rows_p][Hp_p] fp32, rows numbered per player.
//  * showdown tables (built on the host once per board): per player the hands
//    sorted by rank, per card the hands holding it sorted by rank, and per hand
//    its rank position in the opponent's lists.  A terminal then needs one
//    exclusive prefix scan of the opponent's reach in those orders; win, tie
//    and loss masses with card removal are differences of that scan.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mtt {

constexpr int MAXA = 16;           // actions per decision node the solver accepts

struct alignas(16) DNode {
    uint8_t type, player, na, wmask;   // wmask: fold winner bit (active_mask)
    int32_t first;                     // first child (subgame-relative node index)
    int32_t row;                       // first regret row of the acting player
    int32_t reach_src0, reach_src1;    // node whose reach slot holds player 0 / 1 reach here
    float pot, c0, c1;
    int16_t dealt;                     // card dealt by the nearest chance ancestor, -1 if none
    int16_t dealt0;                    // card dealt by the chance ancestor above that one, -1 if none
    int32_t var;                       // showdown table variant of the board this node sees
    int32_t nlive;                     // chance nodes: cards that can be dealt here
};
static_assert(sizeof(DNode) == 48, "DNode is 48 bytes");

struct alignas(16) SubDesc {
    long long node_base;     // into the DNode array
    long long arena_base;    // float offset of the REACH region; CFV region follows (n_nodes*HS)
    long long rs_base0, rs_base1;   // float offsets of R_p (S_p uses the same offsets in S)
    long long tab_base;      // byte offset of the table variants
    long long darena_base;   // double offset of the FP64 best-response arena (3 regions)
    long long range_base;    // float offset of the padded root ranges [Hp0 | Hp1]
    long long hcard_base;    // u16 offset of hand cards [Hp0 | Hp1] (c1 | c2 << 8; 0xFFFF padding)
    int n_nodes;
    int H0, H1, Hp0, Hp1;
    int rows0, rows1;
    int tab_vsize;           // bytes per table variant
    int n_live;              // cards not on the board
    int river;               // 1: single board (variant 0); 0: variants per dealt card(s)
    float pot;               // starting pot (exploitability unit)
    int var_none;            // table variant of the subgame's own board (no card dealt)
    int pad[2];
};

// Table variant layout (bytes), H0/H1 from the descriptor; every block starts
// on a 16-byte boundary so it can be staged with one 1-D bulk copy:
//   IDX0 = u16 sorted0[H0] | u16 cl0[2*H0] | u16 seg0[54]      (opponent lists of player 0)
//   IDX1 = the same for player 1
//   ENT0 = Entry e0[H0] (player-0 hands against player-1 lists), ENT1 = Entry e1[H1]
// One hand against the opponent's lists.  lt / le: position in the
// opponent's rank order of the first hand ranked >= / > this hand;
// ltc1 / lec1 (ltc2 / lec2): the same inside the list of opponent hands
// holding this hand's first (second) card.
struct alignas(4) Entry {
    uint8_t c1, c2, ltc1, lec1, ltc2, lec2;
    uint16_t lt, le;     // lt == 0xFFFF: hand blocked by the dealt card
    int16_t same;        // opponent index of the same combo, -1 if absent
};
static_assert(sizeof(Entry) == 12, "Entry is 12 bytes");

struct TabView {
    const uint16_t* sorted[2];
    const uint16_t* cl[2];
    const uint16_t* seg[2];
    const Entry* ent[2];
};

__host__ __device__ inline int round16(int b) { return (b + 15) & ~15; }
__host__ __device__ inline int tab_idx_bytes(int H) { return round16(2 * (3 * H + 54)); }
__host__ __device__ inline int tab_ent_bytes(int H) { return round16(12 * H); }
__host__ __device__ inline int tab_idx_off(int p, int H0) { return p ? tab_idx_bytes(H0) : 0; }
__host__ __device__ inline int tab_ent_off(int p, int H0, int H1) {
    return tab_idx_bytes(H0) + tab_idx_bytes(H1) + (p ? tab_ent_bytes(H0) : 0);
}
__host__ __device__ inline int tab_variant_bytes(int H0, int H1) {
    return tab_idx_bytes(H0) + tab_idx_bytes(H1) + tab_ent_bytes(H0) + tab_ent_bytes(H1);
}

// Views into one player's index block and entry block (global or shared memory).
__host__ __device__ inline void tab_idx_view(const uint8_t* blk, int H, const uint16_t** sorted,
                                             const uint16_t** cl, const uint16_t** seg) {
    const uint16_t* u = reinterpret_cast<const uint16_t*>(blk);
    *sorted = u;
    *cl = u + H;
    *seg = u + 3 * H;
}

__host__ __device__ inline TabView tab_view(const uint8_t* base, int H0, int H1) {
    TabView v;
    tab_idx_view(base + tab_idx_off(0, H0), H0, &v.sorted[0], &v.cl[0], &v.seg[0]);
    tab_idx_view(base + tab_idx_off(1, H0), H1, &v.sorted[1], &v.cl[1], &v.seg[1]);
    v.ent[0] = reinterpret_cast<const Entry*>(base + tab_ent_off(0, H0, H1));
    v.ent[1] = reinterpret_cast<const Entry*>(base + tab_ent_off(1, H0, H1));
    return v;
}

}  // namespace mtt
