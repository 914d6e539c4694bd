/*
 * mtt_oracle.h — CPU oracle for the MTT-GPU-Solver hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * kernels, used by tests/, __graft_entry__.smoke() and the CPU legs of
 * bench.py as the checker and the timed CPU baseline.  The product library
 * (libmtt_b200.so) never links, loads or calls it.
 *
 * Parity pins:
 *  - orc_score7 / orc_flop_ev / orc_ev_dump reproduce the reference's shipped
 *    data/mtt_ev_dump_1755.bin bit-exactly (tests/golden/ holds slices and a
 *    SHA-256 of the whole file, generated by tests/golden/make_golden.py).
 *  - orc_board_counts, the CFR sweeps, the multiway terminals and the
 *    preflop chain have no reference golden data ("parity unpinned" by
 *    reference artefacts); they follow the cited reference lines and are
 *    cross-checked against the pinned evaluator.
 */
#ifndef MTT_ORACLE_H
#define MTT_ORACLE_H
#include <stdint.h>
#include "../include/mtt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* --- evaluator: src/tools/mtt_ev_dumper.cu:53-83 ------------------------ */
uint32_t orc_score7(const uint8_t cards[7]);
void     orc_eval7_batch(const uint8_t* cards7, uint32_t* out, int64_t n);
/* All C(52,7) hands: category histogram (score>>24, 9 bins) and
 * checksum = sum over hands in colex order of (score * (index+1)) mod 2^64. */
void     orc_enumerate7(uint64_t hist[9], uint64_t* checksum);

/* --- dumper: src/tools/mtt_ev_dumper.cu:17-51,85-116,141-168 ------------- */
int      orc_gen_flops(uint8_t* out /* 1755*4: c1,c2,c3,orbit_weight */);
int      orc_canonical_class(int c1, int c2);
/* One flop through kernel_evaluate_flop_ev (reach NULL = uniform 1/1176). */
void     orc_flop_ev(const uint8_t flop[3], const float* reach0, const float* reach1,
                     float* ev0, float* ev1 /* 1176 each */);
/* Flops [f_begin, f_end) of the canonical list into out[(f-f_begin)][4][2][169]. */
void     orc_ev_dump(int f_begin, int f_end, float* out);

/* --- showdown counts: src/postflop/honest_multistreet_solver.cu:56-86 ----- */
/* nboard 3/4/5; hands H x 2 cards; out[i*H+j] = counts for hero i vs villain j
 * over every completion of the board; conflicting pairs give zeros. */
void     orc_board_counts(const uint8_t* board, int nboard, const uint8_t* hands, int H,
                          int32_t* w, int32_t* t, int32_t* l);

/* --- heads-up CFR sweeps: honest_multistreet_solver.cu:88-249 ------------ */
typedef struct orc_game {
    const mtt_node* nodes;
    int32_t n_nodes;
    int32_t rows[2];
    const uint8_t* board;      /* 5 cards (river) or 4 (turn tree with chance nodes) */
    int32_t nboard;
    int32_t H[2];
    const uint8_t* cards[2];   /* H[p] x 2 hole cards */
    const float* range[2];     /* H[p] root weights */
} orc_game;

#define ORC_ALGO_CFRPLUS 0
#define ORC_ALGO_DCFR    1
#define ORC_SEM_CORRECT   0    /* card removal, ties split, chance / (N-4) */
#define ORC_SEM_REFERENCE 1    /* reference defects: P1 equity inverted, no card removal, chance / (N-2) */

typedef struct orc_cfr_params {
    int32_t iters;
    int32_t algo;
    float   alpha, beta, gamma;
    int32_t semantics;
    int32_t alternate;    /* 0: simultaneous updates (reference kernels), 1: alternating (CFR+ as published) */
    float   avg_power;    /* CFR+ strategy-sum weight t^avg_power */
} orc_cfr_params;

/* Runs iters iterations from zero regrets.  R_p, S_p: [rows_p][H_p].
 * root_cfv_p (optional): last iteration's root counterfactual values. */
int orc_cfr_solve(const orc_game* g, const orc_cfr_params* prm,
                  float* R0, float* R1, float* S0, float* S1,
                  float* root_cfv0, float* root_cfv1);

/* FP64 best response against the average strategies S_p (normalised per
 * hand; uniform where the sum is 0).  out: [0] BR value of P0, [1] BR of P1,
 * [2] EV of P0 under the averages, [3] EV of P1, [4] Z = compatible range
 * mass, [5] exploitability (out[0]+out[1])/2 as a fraction of the starting
 * pot.  Values are per unit of compatible range mass. */
int orc_best_response(const orc_game* g, const float* S0, const float* S1, double out[6]);

/* Root counterfactual values of fixed strategies (FP64).  sigma_p: [rows_p][H_p]
 * behaviour probabilities.  out_cfv_p: [H_p]. ev_out: EV of P0 per unit mass. */
int orc_strategy_values(const orc_game* g, const float* sigma0, const float* sigma1,
                        double* out_cfv0, double* out_cfv1, double* ev_out);

/* EV of P0 in chips when both players play softmax(logits_p) ([rows_p][H_p],
 * per node and hand) with root ranges range_p (FP64 throughout); cfv_p
 * (optional): root counterfactual values [H_p]. */
int orc_softmax_ev(const orc_game* g, const double* logits0, const double* logits1,
                   const double* range0, const double* range1, double* ev0, double* cfv0, double* cfv1);

/* --- four-player river CFR: multiway_4way_engine.cu:41-257 ---------------- */
typedef struct orc_mw_game {
    const mtt_mw_node* nodes;
    int32_t n_nodes;
    int32_t rows[4];
    const uint8_t* board;      /* 5 cards */
    int32_t H;                 /* one combo axis shared by the four players */
    const uint8_t* cards;      /* H x 2 hole cards */
    const float* range[4];
    float bubble[16];
} orc_mw_game;

/* prm: iters, algo (+alpha/beta/gamma), semantics, avg_power (alternate is
 * ignored: the four players update simultaneously).  R[p], S[p]: [rows_p][H];
 * root_cfv (optional): [4][H] of the last iteration; values (optional, [4]):
 * each player's range EV (chips) under the average strategies. */
int orc_mw_solve(const orc_mw_game* g, const orc_cfr_params* prm, float* R[4], float* S[4], float* root_cfv,
                 double* values);
/* The terminal values of node i under the solver's semantics: out [4][H]. */
int orc_mw_terminal_values(const orc_mw_game* g, int i, int sem, const float* const* reach, float* out);
/* The exact four-player showdown (all four hands disjoint) of terminal node i
 * for the given per-player reach vectors ([4] x H): out [4][H], FP64.
 * O(H^3) per hand: small cases only. */
int orc_mw_exact_terminal(const orc_mw_game* g, int i, const float* const* reach, double* out);
/* Malmuth-Harville equity by enumerating the ordered finishers of the m paid places. */
int orc_icm_equity(const double* stacks, int n, const double* payouts, int m, double* out);

/* --- preflop anchor chain: src/preflop/preflop_grid_generator.cu ---------- */
int  orc_pf_combo_class(int c1, int c2);
/* 169 x 169 all-in equities out[h*169+v] (and the integer win/tie counts). */
void orc_pf_allin_matrix(int hc_begin, int hc_end, float* out, int32_t* wins, int32_t* ties);
/* One flop's class-reduced equity matrix out_class[v*169+h] (reference mode). */
void orc_pf_flop_class_matrix(const uint8_t flop[3], float* out_class, float* out_combo);
typedef struct orc_pf_params { int32_t iters; float stack_bb, bubble, dead_pot; } orc_pf_params;
/* DCFR over the closed preflop tree; sums / sigma: [3|3|2|2][192] blocks. */
int orc_pf_dcfr(int nf, const float* flop_weights, const float* class_mats, const float* allin,
                const orc_pf_params* p, float* sums, float* sigma);

#ifdef __cplusplus
}
#endif
#endif
