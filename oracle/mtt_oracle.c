/*
 * mtt_oracle.c — CPU oracle (TEST INFRASTRUCTURE ONLY; see mtt_oracle.h).
 *
 * Plain-C restatement of the reference kernels of MTT-GPU-Solver.  Each
 * function cites the reference lines it follows.  Built with
 * -ffp-contract=off so that the only fused multiply-adds are the explicit
 * fmaf() calls standing in for the contractions nvcc makes in the reference
 * kernels; divisions are IEEE.
 */
#include "mtt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Evaluator: restates fast_7card_score (src/tools/mtt_ev_dumper.cu:53-83),  */
/* identical copies at honest_multistreet_solver.cu:24-54 and               */
/* preflop_grid_generator.cu:47-77.                                          */
/* ------------------------------------------------------------------------ */
static int orc_straight_high(uint32_t m) {          /* f_str, :57-61 */
    for (int r = 12; r >= 4; --r) {
        uint32_t w = 0x1Fu << (r - 4);
        if ((m & w) == w) return r;
    }
    if ((m & 0x100Fu) == 0x100Fu) return 3;
    return -1;
}

uint32_t orc_score7(const uint8_t cards[7]) {
    uint32_t sc[4] = {0, 0, 0, 0}, sm[4] = {0, 0, 0, 0}, rc[13], rm = 0;
    memset(rc, 0, sizeof(rc));
    for (int i = 0; i < 7; ++i) {                       /* :56 */
        int c = cards[i], r = c / 4, s = c % 4;
        sc[s]++; sm[s] |= 1u << r; rc[r]++; rm |= 1u << r;
    }
    for (int s = 0; s < 4; ++s) {                       /* :62-70 */
        if (sc[s] >= 5) {
            int sf = orc_straight_high(sm[s]);
            if (sf != -1) return (8u << 24) | (uint32_t)sf;
            uint32_t score = 5u << 24; int p = 0;
            for (int r = 12; r >= 0 && p < 5; --r)
                if (sm[s] & (1u << r)) { score |= (uint32_t)r << (4 * (4 - p)); ++p; }
            return score;
        }
    }
    int q = -1, t1 = -1, t2 = -1, p1 = -1, p2 = -1;     /* :71-75 */
    for (int r = 12; r >= 0; --r) {
        if (rc[r] == 4) q = r;
        else if (rc[r] == 3) { if (t1 == -1) t1 = r; else if (t2 == -1) t2 = r; }
        else if (rc[r] == 2) { if (p1 == -1) p1 = r; else if (p2 == -1) p2 = r; }
    }
    if (q != -1) return (7u << 24) | ((uint32_t)q << 4);                          /* :76 */
    if (t1 != -1 && (t2 != -1 || p1 != -1))                                        /* :77 */
        return (6u << 24) | ((uint32_t)t1 << 4) | (uint32_t)(t2 != -1 ? t2 : p1);
    int st = orc_straight_high(rm);
    if (st != -1) return (4u << 24) | (uint32_t)st;                                /* :78 */
    if (t1 != -1) return (3u << 24) | ((uint32_t)t1 << 8);                         /* :79 */
    if (p1 != -1 && p2 != -1) return (2u << 24) | ((uint32_t)p1 << 8) | ((uint32_t)p2 << 4); /* :80 */
    if (p1 != -1) return (1u << 24) | ((uint32_t)p1 << 12);                        /* :81 */
    return rm;                                                                     /* :82 */
}

void orc_eval7_batch(const uint8_t* cards7, uint32_t* out, int64_t n) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = orc_score7(cards7 + 7 * i);
}

void orc_enumerate7(uint64_t hist[9], uint64_t* checksum) {
    uint64_t h[9] = {0}, cs = 0;
    /* colex order: largest card outermost; index = sum C(c_i, i+1). */
    #pragma omp parallel
    {
        uint64_t lh[9] = {0}, lcs = 0;
        #pragma omp for schedule(dynamic, 1)
        for (int c6 = 6; c6 < 52; ++c6) {
            /* index of the first subset whose largest card is c6 = C(c6, 7) */
            uint64_t idx = 0;
            { uint64_t b = 1; for (int k = 0; k < 7; ++k) b = b * (uint64_t)(c6 - k) / (uint64_t)(k + 1); idx = b; }
            uint8_t c[7]; c[6] = (uint8_t)c6;
            for (int c5 = 5; c5 < c6; ++c5) { c[5] = (uint8_t)c5;
            for (int c4 = 4; c4 < c5; ++c4) { c[4] = (uint8_t)c4;
            for (int c3 = 3; c3 < c4; ++c3) { c[3] = (uint8_t)c3;
            for (int c2 = 2; c2 < c3; ++c2) { c[2] = (uint8_t)c2;
            for (int c1 = 1; c1 < c2; ++c1) { c[1] = (uint8_t)c1;
            for (int c0 = 0; c0 < c1; ++c0) { c[0] = (uint8_t)c0;
                uint32_t s = orc_score7(c);
                lh[s >> 24]++;
                lcs += (uint64_t)s * (idx + 1);
                ++idx;
            }}}}}}
        }
        #pragma omp critical
        { for (int k = 0; k < 9; ++k) h[k] += lh[k]; cs += lcs; }
    }
    for (int k = 0; k < 9; ++k) hist[k] = h[k];
    *checksum = cs;
}

/* ------------------------------------------------------------------------ */
/* Dumper: flop list (mtt_ev_dumper.cu:34-51), class map (:26-32),          */
/* kernel_evaluate_flop_ev (:85-116), host aggregation (:141-168).          */
/* ------------------------------------------------------------------------ */
int orc_gen_flops(uint8_t* out) {
    int n = 0;
#define MC(r, s) ((uint8_t)((r) * 4 + (s)))
#define PUSH(a, b, c, w) do { out[4*n] = (a); out[4*n+1] = (b); out[4*n+2] = (c); out[4*n+3] = (w); ++n; } while (0)
    for (int r = 12; r >= 0; --r) PUSH(MC(r, 0), MC(r, 1), MC(r, 2), 4);
    for (int rp = 12; rp >= 0; --rp) for (int rk = 12; rk >= 0; --rk) {
        if (rp == rk) continue;
        PUSH(MC(rp, 0), MC(rp, 1), MC(rk, 0), 12);
        PUSH(MC(rp, 0), MC(rp, 1), MC(rk, 2), 12);
    }
    for (int r1 = 12; r1 >= 2; --r1) for (int r2 = r1 - 1; r2 >= 1; --r2) for (int r3 = r2 - 1; r3 >= 0; --r3) {
        PUSH(MC(r1, 0), MC(r2, 0), MC(r3, 0), 4);
        PUSH(MC(r1, 0), MC(r2, 0), MC(r3, 1), 12);
        PUSH(MC(r1, 0), MC(r2, 1), MC(r3, 0), 12);
        PUSH(MC(r1, 1), MC(r2, 0), MC(r3, 0), 12);
        PUSH(MC(r1, 0), MC(r2, 1), MC(r3, 2), 24);
    }
#undef PUSH
#undef MC
    return n;
}

int orc_canonical_class(int c1, int c2) {
    int r1 = c1 / 4, s1 = c1 % 4, r2 = c2 / 4, s2 = c2 % 4;
    int hi = r1 > r2 ? r1 : r2, lo = r1 < r2 ? r1 : r2;
    if (r1 == r2) return 12 - hi;
    int b = (s1 == s2) ? 13 : 91;
    for (int r = 12; r > hi; --r) b += r;
    return b + (hi - 1 - lo);
}

void orc_flop_ev(const uint8_t flop[3], const float* reach0, const float* reach1,
                 float* ev0, float* ev1) {
    uint64_t fm = (1ull << flop[0]) | (1ull << flop[1]) | (1ull << flop[2]);
    uint8_t deck[52]; int nd = 0;
    for (int c = 0; c < 52; ++c) if (!((fm >> c) & 1)) deck[nd++] = (uint8_t)c;   /* :146 */
    uint8_t ac1[1176], ac2[1176]; uint64_t am[1176]; int na = 0;
    for (int c1 = 0; c1 < 52; ++c1) for (int c2 = c1 + 1; c2 < 52; ++c2) {        /* :149-152 */
        uint64_t m = (1ull << c1) | (1ull << c2);
        if (!(m & fm)) { ac1[na] = (uint8_t)c1; ac2[na] = (uint8_t)c2; am[na] = m; ++na; }
    }
    const float uni = 1.0f / 1176.0f;                                              /* :136 */
    #pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < 1176; ++i) {                                               /* :86-116 */
        uint8_t h7[7] = {flop[0], flop[1], flop[2], ac1[i], ac2[i], 0, 0};
        float t0 = 0.0f, t1 = 0.0f;
        for (int j = 0; j < 1176; j += 4) {
            if (am[i] & am[j]) continue;
            uint8_t v7[7] = {flop[0], flop[1], flop[2], ac1[j], ac2[j], 0, 0};
            uint64_t dead = am[i] | am[j];
            int wins = 0, ties = 0, total = 0;
            for (int r1 = 0; r1 < 47; r1 += 2) {
                uint8_t turn = deck[r1];
                if ((dead >> turn) & 1) continue;
                h7[5] = turn; v7[5] = turn;
                for (int r2 = r1 + 1; r2 < 47; r2 += 3) {
                    uint8_t river = deck[r2];
                    if ((dead >> river) & 1) continue;
                    h7[6] = river; v7[6] = river;
                    uint32_t sh = orc_score7(h7), sv = orc_score7(v7);
                    if (sh > sv) wins += 2; else if (sh == sv) ties += 1;
                    total += 2;
                }
            }
            if (total > 0) {
                float eq = (float)(wins + ties) / (float)total;
                float r1j = reach1 ? reach1[j] : uni, r0j = reach0 ? reach0[j] : uni;
                t0 = fmaf(r1j, fmaf(eq, 2.0f, -1.0f), t0);          /* :111, contracted */
                t1 = fmaf(r0j, fmaf(1.0f - eq, 2.0f, -1.0f), t1);   /* :112, contracted */
            }
        }
        ev0[i] = t0; ev1[i] = t1;
    }
}

void orc_ev_dump(int f_begin, int f_end, float* out) {
    uint8_t flops[1755 * 4];
    orc_gen_flops(flops);
    float* ev0 = (float*)malloc(1176 * sizeof(float));
    float* ev1 = (float*)malloc(1176 * sizeof(float));
    for (int f = f_begin; f < f_end; ++f) {
        const uint8_t* fl = flops + 4 * f;
        uint64_t fm = (1ull << fl[0]) | (1ull << fl[1]) | (1ull << fl[2]);
        int cls[1176], na = 0;
        for (int c1 = 0; c1 < 52; ++c1) for (int c2 = c1 + 1; c2 < 52; ++c2) {
            uint64_t m = (1ull << c1) | (1ull << c2);
            if (!(m & fm)) cls[na++] = orc_canonical_class(c1, c2);
        }
        orc_flop_ev(fl, NULL, NULL, ev0, ev1);
        float* o = out + (size_t)(f - f_begin) * 4 * 2 * 169;
        memset(o, 0, 4 * 2 * 169 * sizeof(float));
        for (int scen = 0; scen < 4; ++scen) {                                     /* :160-168 */
            float mult = 1.0f + 0.1f * (float)scen;
            float* b = o + scen * 2 * 169;
            for (int c = 0; c < 1176; ++c) {
                b[cls[c]]       = b[cls[c]]       + ev0[c] * mult;
                b[169 + cls[c]] = b[169 + cls[c]] + ev1[c] * mult;
            }
        }
    }
    free(ev0); free(ev1);
}

/* ------------------------------------------------------------------------ */
/* Showdown counts: kernel_gen_49_turn_matrices (honest:56-86) generalised   */
/* to 3/4/5-card boards by exact enumeration of the missing board cards.     */
/* ------------------------------------------------------------------------ */
void orc_board_counts(const uint8_t* board, int nboard, const uint8_t* hands, int H,
                      int32_t* w, int32_t* t, int32_t* l) {
    uint64_t bm = 0;
    for (int k = 0; k < nboard; ++k) bm |= 1ull << board[k];
    uint8_t rest[52]; int nr = 0;
    for (int c = 0; c < 52; ++c) if (!((bm >> c) & 1)) rest[nr++] = (uint8_t)c;
    int need = 5 - nboard;
    /* completions: list of (c_a, c_b) (c_b = 255 when need == 1; none when 0) */
    int ncomp = need == 0 ? 1 : need == 1 ? nr : nr * (nr - 1) / 2;
    uint8_t* ca = (uint8_t*)malloc((size_t)ncomp), *cb = (uint8_t*)malloc((size_t)ncomp);
    {
        int k = 0;
        if (need == 0) { ca[0] = 255; cb[0] = 255; }
        else if (need == 1) for (int a = 0; a < nr; ++a) { ca[k] = rest[a]; cb[k] = 255; ++k; }
        else for (int a = 0; a < nr; ++a) for (int b = a + 1; b < nr; ++b) { ca[k] = rest[a]; cb[k] = rest[b]; ++k; }
    }
    uint32_t* sc = (uint32_t*)malloc((size_t)ncomp * (size_t)H * sizeof(uint32_t));
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < ncomp; ++k) {
        uint8_t c7[7];
        for (int b = 0; b < nboard; ++b) c7[b] = board[b];
        int nb = nboard;
        if (ca[k] != 255) c7[nb++] = ca[k];
        if (cb[k] != 255) c7[nb++] = cb[k];
        for (int h = 0; h < H; ++h) {
            c7[5] = hands[2 * h]; c7[6] = hands[2 * h + 1];
            sc[(size_t)k * H + h] = orc_score7(c7);
        }
    }
    #pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < H; ++i) {
        uint64_t mi = (1ull << hands[2 * i]) | (1ull << hands[2 * i + 1]);
        for (int j = 0; j < H; ++j) {
            uint64_t mj = (1ull << hands[2 * j]) | (1ull << hands[2 * j + 1]);
            int32_t W = 0, T = 0, L = 0;
            if (!(mi & mj) && !(mi & bm) && !(mj & bm)) {
                uint64_t dead = mi | mj;
                for (int k = 0; k < ncomp; ++k) {
                    if (ca[k] != 255 && ((dead >> ca[k]) & 1)) continue;
                    if (cb[k] != 255 && ((dead >> cb[k]) & 1)) continue;
                    uint32_t si = sc[(size_t)k * H + i], sj = sc[(size_t)k * H + j];
                    if (si > sj) ++W; else if (si == sj) ++T; else ++L;
                }
            }
            w[(size_t)i * H + j] = W; t[(size_t)i * H + j] = T; l[(size_t)i * H + j] = L;
        }
    }
    free(sc); free(ca); free(cb);
}

/* ------------------------------------------------------------------------ */
/* Heads-up CFR: kernel_forward_sweep (honest:88-126), kernel_evaluate_      */
/* terminals (:128-196), kernel_backward_sweep (:198-249), with the DCFR     */
/* discounting of kernel_dcfr_step (preflop_grid_generator.cu:387-410) in    */
/* the standard discount-then-add form.                                      */
/* ------------------------------------------------------------------------ */
typedef struct orc_ctx {
    const orc_game* g;
    int n;
    int* parent;
    uint64_t* dmask;     /* cards dealt at and above each node (chance children carry their card) */
    int* sidx;           /* showdown nodes: row of score[] for the node's 5-card board, else -1 */
    uint64_t* hmask[2];  /* per hand card mask */
    uint32_t* score[2];  /* [n_boards][H_p]: score on each distinct showdown board */
    int n_boards;
} orc_ctx;

static int popc64(uint64_t x) { int k = 0; while (x) { x &= x - 1; ++k; } return k; }

/* Cards that a chance node can deal: not on the board, not dealt above. */
static int orc_nlive(const orc_ctx* c, int node) {
    return 52 - c->g->nboard - popc64(c->dmask[node]);
}

static int orc_ctx_init(orc_ctx* c, const orc_game* g) {
    memset(c, 0, sizeof(*c));
    c->g = g; c->n = g->n_nodes;
    if (g->nboard < 3 || g->nboard > 5) return MTT_ERR_INVALID;
    c->parent = (int*)malloc(sizeof(int) * (size_t)c->n);
    c->dmask = (uint64_t*)calloc((size_t)c->n, sizeof(uint64_t));
    c->sidx = (int*)malloc(sizeof(int) * (size_t)c->n);
    for (int i = 0; i < c->n; ++i) { c->parent[i] = -1; c->sidx[i] = -1; }
    for (int i = 0; i < c->n; ++i) {
        const mtt_node* nd = &g->nodes[i];
        if (nd->type == MTT_NODE_DECISION || nd->type == MTT_NODE_CHANCE)
            for (int a = 0; a < nd->num_actions; ++a) c->parent[nd->children_offset + a] = i;
    }
    for (int i = 0; i < c->n; ++i) {   /* BFS order: parents first */
        int p = c->parent[i];
        if (p < 0) continue;
        c->dmask[i] = c->dmask[p];
        if (g->nodes[p].type == MTT_NODE_CHANCE) c->dmask[i] |= 1ull << g->nodes[i].turn_idx;
    }
    /* distinct showdown boards (open addressing on the dealt-card mask) */
    const int tsize = 1 << 14;
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * tsize);
    int* vals = (int*)malloc(sizeof(int) * tsize);
    for (int k = 0; k < tsize; ++k) vals[k] = -1;
    uint64_t* masks = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)c->n);
    for (int i = 0; i < c->n; ++i) {
        if (g->nodes[i].type != MTT_NODE_SHOWDOWN) continue;
        uint64_t m = c->dmask[i];
        unsigned hsh = (unsigned)((m * 0x9E3779B97F4A7C15ull) >> 50) & (tsize - 1);
        while (vals[hsh] >= 0 && keys[hsh] != m) hsh = (hsh + 1) & (tsize - 1);
        if (vals[hsh] < 0) { keys[hsh] = m; vals[hsh] = c->n_boards; masks[c->n_boards++] = m; }
        c->sidx[i] = vals[hsh];
    }
    free(keys); free(vals);
    for (int p = 0; p < 2; ++p) {
        int H = g->H[p];
        c->hmask[p] = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(H > 0 ? H : 1));
        c->score[p] = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(c->n_boards > 0 ? c->n_boards : 1) *
                                        (size_t)(H > 0 ? H : 1));
        for (int h = 0; h < H; ++h)
            c->hmask[p][h] = (1ull << g->cards[p][2 * h]) | (1ull << g->cards[p][2 * h + 1]);
        for (int b = 0; b < c->n_boards; ++b) {
            uint8_t c7[7];
            int k = 0;
            for (; k < g->nboard; ++k) c7[k] = g->board[k];
            for (int x = 0; x < 52 && k < 5; ++x) if ((masks[b] >> x) & 1ull) c7[k++] = (uint8_t)x;
            for (int h = 0; h < H; ++h) {
                c7[5] = g->cards[p][2 * h]; c7[6] = g->cards[p][2 * h + 1];
                c->score[p][(size_t)b * H + h] = orc_score7(c7);
            }
        }
    }
    free(masks);
    return MTT_OK;
}

static void orc_ctx_free(orc_ctx* c) {
    free(c->parent); free(c->dmask); free(c->sidx);
    for (int p = 0; p < 2; ++p) { free(c->hmask[p]); free(c->score[p]); }
}

/* Terminal values for player q against opponent reach ro (double math).    */
/* sem: ORC_SEM_CORRECT or ORC_SEM_REFERENCE (honest:134-195 defects).      */
static void orc_terminal_values(const orc_ctx* c, int node, int q, const double* ro,
                                int sem, double* out) {
    const orc_game* g = c->g;
    const mtt_node* nd = &g->nodes[node];
    int o = 1 - q, Hq = g->H[q], Ho = g->H[o];
    uint64_t dm = c->dmask[node];   /* cards dealt above: hands holding one are blocked */
    if (nd->type == MTT_NODE_FOLD) {
        int winner = (nd->active_mask == 1) ? 0 : 1;                       /* :135 */
        double payoff = (q == winner) ? (double)nd->pot_size - (double)nd->committed[q]
                                      : -(double)nd->committed[q];           /* :163-164 */
        double tot = 0.0;
        for (int j = 0; j < Ho; ++j) tot += ro[j];
        for (int h = 0; h < Hq; ++h) {
            double m;
            if (c->hmask[q][h] & dm) { out[h] = 0.0; continue; }   /* blocked by a dealt card */
            if (sem == ORC_SEM_REFERENCE) m = tot;
            else {
                m = 0.0;
                uint64_t mh = c->hmask[q][h] | dm;
                for (int j = 0; j < Ho; ++j) if (!(c->hmask[o][j] & mh)) m += ro[j];
            }
            out[h] = payoff * m;
        }
        return;
    }
    /* showdown: honest:170-195 */
    const uint32_t* sq = c->score[q] + (size_t)c->sidx[node] * Hq;
    const uint32_t* so = c->score[o] + (size_t)c->sidx[node] * Ho;
    double gain = (double)nd->pot_size - (double)nd->committed[q];
    double loss = -(double)nd->committed[q];
    double tie = 0.5 * (double)nd->pot_size - (double)nd->committed[q];
    for (int h = 0; h < Hq; ++h) {
        double acc = 0.0;
        uint64_t mh = c->hmask[q][h];
        if (sem == ORC_SEM_CORRECT) {
            if (mh & dm) { out[h] = 0.0; continue; }
            for (int j = 0; j < Ho; ++j) {
                if (c->hmask[o][j] & (mh | dm)) continue;
                double v = sq[h] > so[j] ? gain : (sq[h] == so[j] ? tie : loss);
                acc += ro[j] * v;
            }
        } else {
            for (int j = 0; j < Ho; ++j) {
                int compat = !(c->hmask[o][j] & (mh | dm)) && !(mh & dm);
                double eq = compat ? (sq[h] > so[j] ? 1.0 : (sq[h] == so[j] ? 0.5 : 0.0)) : 0.0;
                if (q == 1) eq = 1.0 - eq;            /* :184-186 P1 uses 1 - eq(tid vs j) */
                acc += ro[j] * (eq * gain + (1.0 - eq) * loss);
            }
        }
        out[h] = acc;
    }
}

int orc_cfr_solve(const orc_game* g, const orc_cfr_params* prm,
                  float* R0, float* R1, float* S0, float* S1,
                  float* root_cfv0, float* root_cfv1) {
    orc_ctx c;
    int st = orc_ctx_init(&c, g);
    if (st) return st;
    int n = g->n_nodes, H[2] = {g->H[0], g->H[1]};
    float* R[2] = {R0, R1};
    float* S[2] = {S0, S1};
    for (int p = 0; p < 2; ++p) {
        memset(R[p], 0, sizeof(float) * (size_t)g->rows[p] * (size_t)H[p]);
        memset(S[p], 0, sizeof(float) * (size_t)g->rows[p] * (size_t)H[p]);
    }
    float* reach[2]; float* cfv[2]; float* sig[2];
    for (int p = 0; p < 2; ++p) {
        reach[p] = (float*)calloc((size_t)n * (size_t)H[p], sizeof(float));
        cfv[p] = (float*)calloc((size_t)n * (size_t)H[p], sizeof(float));
        sig[p] = (float*)calloc((size_t)g->rows[p] * (size_t)H[p] + 1, sizeof(float));
    }
    int Hmax = H[0] > H[1] ? H[0] : H[1];
    double* ro = (double*)malloc(sizeof(double) * (size_t)(Hmax + 1));
    double* tv = (double*)malloc(sizeof(double) * (size_t)(Hmax + 1));

    /* Simultaneous updates (the reference kernels: one forward and one
     * backward sweep update both players) or alternating updates (CFR+ as
     * published: P0's pass, then P1's pass against P0's new strategy). */
    const int n_pass = prm->alternate ? 2 : 1;
    for (int t = 1; t <= prm->iters; ++t) {
        float w_lin = (float)pow((double)t, (double)prm->avg_power);
        double tm1 = (double)(t - 1);
        float dpos = (float)(pow(tm1, (double)prm->alpha) / (pow(tm1, (double)prm->alpha) + 1.0));
        float dneg = (float)(pow(tm1, (double)prm->beta) / (pow(tm1, (double)prm->beta) + 1.0));
        float dstr = (float)pow(tm1 / (double)t, (double)prm->gamma);
        for (int pass = 0; pass < n_pass; ++pass) {
        const int upd = prm->alternate ? (1 << pass) : 3;    /* bit p: player p is updated */
        /* forward (parents before children) */
        for (int p = 0; p < 2; ++p) memcpy(reach[p], g->range[p], sizeof(float) * (size_t)H[p]);
        for (int i = 0; i < n; ++i) {
            const mtt_node* nd = &g->nodes[i];
            if (nd->type == MTT_NODE_DECISION) {
                int p = nd->player, o = 1 - p, A = nd->num_actions, row = nd->infoset_offset;
                for (int h = 0; h < H[p]; ++h) {
                    float pos[16], sum = 0.0f;
                    for (int a = 0; a < A; ++a) {
                        pos[a] = fmaxf(R[p][(size_t)(row + a) * H[p] + h], 0.0f);
                        sum += pos[a];
                    }
                    float rp = reach[p][(size_t)i * H[p] + h];
                    for (int a = 0; a < A; ++a) {
                        float s = (sum > 1e-7f) ? pos[a] / sum : 1.0f / (float)A;   /* :117 */
                        sig[p][(size_t)(row + a) * H[p] + h] = s;
                        reach[p][(size_t)(nd->children_offset + a) * H[p] + h] = rp * s;
                        if (!((upd >> p) & 1)) continue;
                        float* sp = &S[p][(size_t)(row + a) * H[p] + h];
                        if (prm->algo == ORC_ALGO_DCFR) *sp = fmaf(rp, s, *sp * dstr);
                        else *sp = fmaf(w_lin * rp, s, *sp);                          /* :244 */
                    }
                }
                for (int a = 0; a < A; ++a)
                    memcpy(&reach[o][(size_t)(nd->children_offset + a) * H[o]],
                           &reach[o][(size_t)i * H[o]], sizeof(float) * (size_t)H[o]);
            } else if (nd->type == MTT_NODE_CHANCE) {                                /* :97-104 */
                for (int a = 0; a < nd->num_actions; ++a) {
                    int ch = nd->children_offset + a;
                    uint64_t cm = 1ull << g->nodes[ch].turn_idx;
                    for (int p = 0; p < 2; ++p)
                        for (int h = 0; h < H[p]; ++h)
                            reach[p][(size_t)ch * H[p] + h] =
                                (c.hmask[p][h] & cm) ? 0.0f : reach[p][(size_t)i * H[p] + h];
                }
            }
        }
        /* terminals */
        for (int i = 0; i < n; ++i) {
            const mtt_node* nd = &g->nodes[i];
            if (nd->type != MTT_NODE_FOLD && nd->type != MTT_NODE_SHOWDOWN) continue;
            for (int q = 0; q < 2; ++q) {
                if (!((upd >> q) & 1)) continue;
                int o = 1 - q;
                for (int j = 0; j < H[o]; ++j) ro[j] = reach[o][(size_t)i * H[o] + j];
                orc_terminal_values(&c, i, q, ro, prm->semantics, tv);
                for (int h = 0; h < H[q]; ++h) cfv[q][(size_t)i * H[q] + h] = (float)tv[h];
            }
        }
        /* backward (children before parents) */
        for (int i = n - 1; i >= 0; --i) {
            const mtt_node* nd = &g->nodes[i];
            if (nd->type == MTT_NODE_DECISION) {                                     /* :220-246 */
                int p = nd->player, o = 1 - p, A = nd->num_actions, row = nd->infoset_offset;
                if ((upd >> p) & 1) {
                    for (int h = 0; h < H[p]; ++h) {
                        float v = 0.0f;
                        for (int a = 0; a < A; ++a)
                            v = fmaf(sig[p][(size_t)(row + a) * H[p] + h],
                                     cfv[p][(size_t)(nd->children_offset + a) * H[p] + h], v);
                        cfv[p][(size_t)i * H[p] + h] = v;
                        for (int a = 0; a < A; ++a) {
                            float qa = cfv[p][(size_t)(nd->children_offset + a) * H[p] + h];
                            float* rr = &R[p][(size_t)(row + a) * H[p] + h];
                            float inst = qa - v;
                            if (prm->algo == ORC_ALGO_DCFR) {
                                float disc = *rr * (*rr > 0.0f ? dpos : dneg);
                                *rr = disc + inst;
                            } else {
                                *rr = fmaxf(0.0f, *rr + inst);                      /* :243 */
                            }
                        }
                    }
                }
                if ((upd >> o) & 1) {
                    for (int h = 0; h < H[o]; ++h) {
                        float so = 0.0f;
                        for (int a = 0; a < A; ++a) so += cfv[o][(size_t)(nd->children_offset + a) * H[o] + h];
                        cfv[o][(size_t)i * H[o] + h] = so;
                    }
                }
            } else if (nd->type == MTT_NODE_CHANCE) {                                /* :205-219 */
                const float chance_div = (float)(orc_nlive(&c, i) - (prm->semantics == ORC_SEM_REFERENCE ? 2 : 4));
                for (int p = 0; p < 2; ++p) {
                    if (!((upd >> p) & 1)) continue;
                    for (int h = 0; h < H[p]; ++h) {
                        float acc = 0.0f;
                        for (int a = 0; a < nd->num_actions; ++a) {
                            int ch = nd->children_offset + a;
                            if (c.hmask[p][h] & (1ull << g->nodes[ch].turn_idx)) continue;
                            acc += cfv[p][(size_t)ch * H[p] + h];
                        }
                        cfv[p][(size_t)i * H[p] + h] = acc / chance_div;   /* N-2 or N-4, N per node */
                    }
                }
            }
        }
        }
    }
    if (root_cfv0) memcpy(root_cfv0, cfv[0], sizeof(float) * (size_t)H[0]);
    if (root_cfv1) memcpy(root_cfv1, cfv[1], sizeof(float) * (size_t)H[1]);
    for (int p = 0; p < 2; ++p) { free(reach[p]); free(cfv[p]); free(sig[p]); }
    free(ro); free(tv);
    orc_ctx_free(&c);
    return MTT_OK;
}

/* Shared FP64 pass: values of both players when each plays `pol_p`
 * (behaviour probabilities), plus best-response values. */
static int orc_values_fp64(const orc_game* g, const double* pol0, const double* pol1,
                           double* br_root0, double* br_root1,
                           double* ev_root0, double* ev_root1, double* Z, const double* const* rng) {
    orc_ctx c;
    int st = orc_ctx_init(&c, g);
    if (st) return st;
    int n = g->n_nodes, H[2] = {g->H[0], g->H[1]};
    const double* pol[2] = {pol0, pol1};
    double *reach[2], *br[2], *ev[2];
    for (int p = 0; p < 2; ++p) {
        reach[p] = (double*)calloc((size_t)n * (size_t)H[p] + 1, sizeof(double));
        br[p] = (double*)calloc((size_t)n * (size_t)H[p] + 1, sizeof(double));
        ev[p] = (double*)calloc((size_t)n * (size_t)H[p] + 1, sizeof(double));
        for (int h = 0; h < H[p]; ++h) reach[p][h] = rng ? rng[p][h] : (double)g->range[p][h];
    }
    int Hmax = H[0] > H[1] ? H[0] : H[1];
    double* tv = (double*)malloc(sizeof(double) * (size_t)(Hmax + 1));
    for (int i = 0; i < n; ++i) {
        const mtt_node* nd = &g->nodes[i];
        if (nd->type == MTT_NODE_DECISION) {
            int p = nd->player, o = 1 - p;
            for (int a = 0; a < nd->num_actions; ++a) {
                int ch = nd->children_offset + a;
                for (int h = 0; h < H[p]; ++h)
                    reach[p][(size_t)ch * H[p] + h] = reach[p][(size_t)i * H[p] + h] *
                        pol[p][(size_t)(nd->infoset_offset + a) * H[p] + h];
                memcpy(&reach[o][(size_t)ch * H[o]], &reach[o][(size_t)i * H[o]], sizeof(double) * (size_t)H[o]);
            }
        } else if (nd->type == MTT_NODE_CHANCE) {
            for (int a = 0; a < nd->num_actions; ++a) {
                int ch = nd->children_offset + a;
                uint64_t cm = 1ull << g->nodes[ch].turn_idx;
                for (int p = 0; p < 2; ++p)
                    for (int h = 0; h < H[p]; ++h)
                        reach[p][(size_t)ch * H[p] + h] = (c.hmask[p][h] & cm) ? 0.0 : reach[p][(size_t)i * H[p] + h];
            }
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        const mtt_node* nd = &g->nodes[i];
        if (nd->type == MTT_NODE_FOLD || nd->type == MTT_NODE_SHOWDOWN) {
            for (int q = 0; q < 2; ++q) {
                int o = 1 - q;
                orc_terminal_values(&c, i, q, &reach[o][(size_t)i * H[o]], ORC_SEM_CORRECT, tv);
                for (int h = 0; h < H[q]; ++h) {
                    br[q][(size_t)i * H[q] + h] = tv[h];
                    ev[q][(size_t)i * H[q] + h] = tv[h];
                }
            }
        } else if (nd->type == MTT_NODE_DECISION) {
            int p = nd->player, o = 1 - p;
            for (int h = 0; h < H[p]; ++h) {
                double best = -1e300, v = 0.0;
                for (int a = 0; a < nd->num_actions; ++a) {
                    int ch = nd->children_offset + a;
                    double b = br[p][(size_t)ch * H[p] + h];
                    if (b > best) best = b;
                    v += pol[p][(size_t)(nd->infoset_offset + a) * H[p] + h] * ev[p][(size_t)ch * H[p] + h];
                }
                br[p][(size_t)i * H[p] + h] = best;
                ev[p][(size_t)i * H[p] + h] = v;
            }
            for (int h = 0; h < H[o]; ++h) {
                double sb = 0.0, se = 0.0;
                for (int a = 0; a < nd->num_actions; ++a) {
                    int ch = nd->children_offset + a;
                    sb += br[o][(size_t)ch * H[o] + h];
                    se += ev[o][(size_t)ch * H[o] + h];
                }
                br[o][(size_t)i * H[o] + h] = sb;
                ev[o][(size_t)i * H[o] + h] = se;
            }
        } else if (nd->type == MTT_NODE_CHANCE) {
            double div = (double)(orc_nlive(&c, i) - 4);
            for (int p = 0; p < 2; ++p)
                for (int h = 0; h < H[p]; ++h) {
                    double sb = 0.0, se = 0.0;
                    for (int a = 0; a < nd->num_actions; ++a) {
                        int ch = nd->children_offset + a;
                        if (c.hmask[p][h] & (1ull << g->nodes[ch].turn_idx)) continue;
                        sb += br[p][(size_t)ch * H[p] + h];
                        se += ev[p][(size_t)ch * H[p] + h];
                    }
                    br[p][(size_t)i * H[p] + h] = sb / div;
                    ev[p][(size_t)i * H[p] + h] = se / div;
                }
        }
    }
    /* compatible range mass */
    double z = 0.0;
    for (int h = 0; h < H[0]; ++h) {
        double m = 0.0;
        for (int j = 0; j < H[1]; ++j)
            if (!(c.hmask[0][h] & c.hmask[1][j])) m += rng ? rng[1][j] : (double)g->range[1][j];
        z += (rng ? rng[0][h] : (double)g->range[0][h]) * m;
    }
    *Z = z;
    if (br_root0) memcpy(br_root0, br[0], sizeof(double) * (size_t)H[0]);
    if (br_root1) memcpy(br_root1, br[1], sizeof(double) * (size_t)H[1]);
    if (ev_root0) memcpy(ev_root0, ev[0], sizeof(double) * (size_t)H[0]);
    if (ev_root1) memcpy(ev_root1, ev[1], sizeof(double) * (size_t)H[1]);
    for (int p = 0; p < 2; ++p) { free(reach[p]); free(br[p]); free(ev[p]); }
    free(tv);
    orc_ctx_free(&c);
    return MTT_OK;
}

static double* orc_avg_policy(const orc_game* g, int p, const float* S) {
    int H = g->H[p];
    double* pol = (double*)calloc((size_t)g->rows[p] * (size_t)H + 1, sizeof(double));
    for (int i = 0; i < g->n_nodes; ++i) {
        const mtt_node* nd = &g->nodes[i];
        if (nd->type != MTT_NODE_DECISION || nd->player != p) continue;
        int A = nd->num_actions, row = nd->infoset_offset;
        for (int h = 0; h < H; ++h) {
            double sum = 0.0;
            for (int a = 0; a < A; ++a) sum += (double)S[(size_t)(row + a) * H + h];
            for (int a = 0; a < A; ++a)
                pol[(size_t)(row + a) * H + h] = sum > 0.0 ? (double)S[(size_t)(row + a) * H + h] / sum : 1.0 / A;
        }
    }
    return pol;
}

int orc_best_response(const orc_game* g, const float* S0, const float* S1, double out[6]) {
    double* pol0 = orc_avg_policy(g, 0, S0);
    double* pol1 = orc_avg_policy(g, 1, S1);
    int H0 = g->H[0], H1 = g->H[1];
    double* b0 = (double*)malloc(sizeof(double) * (size_t)(H0 + 1));
    double* b1 = (double*)malloc(sizeof(double) * (size_t)(H1 + 1));
    double* e0 = (double*)malloc(sizeof(double) * (size_t)(H0 + 1));
    double* e1 = (double*)malloc(sizeof(double) * (size_t)(H1 + 1));
    double Z = 0.0;
    int st = orc_values_fp64(g, pol0, pol1, b0, b1, e0, e1, &Z, NULL);
    if (st == MTT_OK) {
        double br0 = 0, br1 = 0, ev0 = 0, ev1 = 0;
        for (int h = 0; h < H0; ++h) { br0 += g->range[0][h] * b0[h]; ev0 += g->range[0][h] * e0[h]; }
        for (int h = 0; h < H1; ++h) { br1 += g->range[1][h] * b1[h]; ev1 += g->range[1][h] * e1[h]; }
        double zz = Z > 0 ? Z : 1.0;
        out[0] = br0 / zz; out[1] = br1 / zz; out[2] = ev0 / zz; out[3] = ev1 / zz; out[4] = Z;
        out[5] = 0.5 * (out[0] + out[1]) / (double)g->nodes[0].pot_size;
    }
    free(pol0); free(pol1); free(b0); free(b1); free(e0); free(e1);
    return st;
}

int orc_strategy_values(const orc_game* g, const float* sigma0, const float* sigma1,
                        double* out_cfv0, double* out_cfv1, double* ev_out) {
    int rows0 = g->rows[0], rows1 = g->rows[1];
    double* pol0 = (double*)malloc(sizeof(double) * ((size_t)rows0 * (size_t)g->H[0] + 1));
    double* pol1 = (double*)malloc(sizeof(double) * ((size_t)rows1 * (size_t)g->H[1] + 1));
    for (size_t k = 0; k < (size_t)rows0 * (size_t)g->H[0]; ++k) pol0[k] = sigma0[k];
    for (size_t k = 0; k < (size_t)rows1 * (size_t)g->H[1]; ++k) pol1[k] = sigma1[k];
    double Z = 0.0;
    int st = orc_values_fp64(g, pol0, pol1, NULL, NULL, out_cfv0, out_cfv1, &Z, NULL);
    if (st == MTT_OK && ev_out) {
        double ev = 0.0;
        for (int h = 0; h < g->H[0]; ++h) ev += (double)g->range[0][h] * out_cfv0[h];
        *ev_out = ev;
    }
    free(pol0); free(pol1);
    return st;
}

/* Differentiable-EV oracle: both players play softmax(logits) per node and
 * hand; FP64 throughout.  EV0 = sum over hands of range0 * cfv0(root) in
 * chips (the values of orc_values_fp64, i.e. kernel_evaluate_terminals and
 * kernel_backward_sweep of honest_multistreet_solver.cu:128-249 with card
 * removal). */
int orc_softmax_ev(const orc_game* g, const double* logits0, const double* logits1,
                   const double* range0, const double* range1, double* ev0, double* cfv0, double* cfv1) {
    const double* lg[2] = {logits0, logits1};
    double* pol[2];
    for (int p = 0; p < 2; ++p) {
        const int H = g->H[p];
        pol[p] = (double*)calloc((size_t)g->rows[p] * (size_t)H + 1, sizeof(double));
        for (int i = 0; i < g->n_nodes; ++i) {
            const mtt_node* nd = &g->nodes[i];
            if (nd->type != MTT_NODE_DECISION || nd->player != p) continue;
            const int A = nd->num_actions, r0 = nd->infoset_offset;
            for (int h = 0; h < H; ++h) {
                double m = -1e300, den = 0.0;
                for (int a = 0; a < A; ++a) { double l = lg[p][(size_t)(r0 + a) * H + h]; if (l > m) m = l; }
                for (int a = 0; a < A; ++a) den += exp(lg[p][(size_t)(r0 + a) * H + h] - m);
                for (int a = 0; a < A; ++a)
                    pol[p][(size_t)(r0 + a) * H + h] = exp(lg[p][(size_t)(r0 + a) * H + h] - m) / den;
            }
        }
    }
    const double* rng[2] = {range0, range1};
    double* c0 = (double*)malloc(sizeof(double) * ((size_t)g->H[0] + 1));
    double* c1 = (double*)malloc(sizeof(double) * ((size_t)g->H[1] + 1));
    double Z = 0.0;
    int st = orc_values_fp64(g, pol[0], pol[1], NULL, NULL, c0, c1, &Z, rng);
    if (st == MTT_OK) {
        double ev = 0.0;
        for (int h = 0; h < g->H[0]; ++h) ev += range0[h] * c0[h];
        if (ev0) *ev0 = ev;
        if (cfv0) memcpy(cfv0, c0, sizeof(double) * (size_t)g->H[0]);
        if (cfv1) memcpy(cfv1, c1, sizeof(double) * (size_t)g->H[1]);
    }
    free(c0); free(c1); free(pol[0]); free(pol[1]);
    return st;
}

/* ------------------------------------------------------------------------ */
/* Four-player river CFR: restates kernel_4way_forward_sweep,               */
/* kernel_4way_evaluate_terminals and kernel_4way_backward_cfr_plus          */
/* (src/postflop/multiway_4way_engine.cu:41-257) with simultaneous updates;  */
/* FP32 storage, terminal values in FP64 rounded to float.                   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int H, n;
    int* pos; int* gs; int* ge;      /* rank position, rank-group bounds per hand */
    uint32_t* sc;                    /* score per hand */
    uint64_t* mask;                  /* hole-card bit mask per hand */
} orc_mw_ctx;

static void orc_mw_ranks(const orc_mw_game* g, orc_mw_ctx* c) {
    int H = g->H;
    uint32_t* sc = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(H + 1));
    int* ord = (int*)malloc(sizeof(int) * (size_t)(H + 1));
    c->mask = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(H + 1));
    for (int h = 0; h < H; ++h) {
        uint8_t cards[7] = {g->board[0], g->board[1], g->board[2], g->board[3], g->board[4],
                            g->cards[2 * h], g->cards[2 * h + 1]};
        sc[h] = orc_score7(cards);
        ord[h] = h;
        c->mask[h] = (1ull << g->cards[2 * h]) | (1ull << g->cards[2 * h + 1]);
    }
    /* stable insertion sort by score (ties keep index order) */
    for (int i = 1; i < H; ++i) {
        int x = ord[i], j = i - 1;
        while (j >= 0 && sc[ord[j]] > sc[x]) { ord[j + 1] = ord[j]; --j; }
        ord[j + 1] = x;
    }
    c->pos = (int*)malloc(sizeof(int) * (size_t)(H + 1));
    c->gs = (int*)malloc(sizeof(int) * (size_t)(H + 1));
    c->ge = (int*)malloc(sizeof(int) * (size_t)(H + 1));
    for (int i = 0; i < H;) {
        int j = i;
        while (j < H && sc[ord[j]] == sc[ord[i]]) ++j;
        for (int k = i; k < j; ++k) { c->pos[ord[k]] = k; c->gs[ord[k]] = i; c->ge[ord[k]] = j; }
        i = j;
    }
    c->H = H;
    c->sc = sc;
    free(ord);
}

static void orc_mw_free(orc_mw_ctx* c) { free(c->pos); free(c->gs); free(c->ge); free(c->sc); free(c->mask); }

/* Terminal values of all four players at node i (kernel_4way_evaluate_terminals).
 * Reference semantics: the reference's rank-position CDFs, no ties, no card
 * removal.  Correct semantics: each opponent's mass is counted only over the
 * hands that share no card with the hero's hand (the hero's own cards are
 * removed from every opponent's range; opponents are not conditioned on one
 * another), below (L), equal to (E) and in total (W); equal hands split the
 * pot.  Both by direct FP64 sums. */
static void orc_mw_terminal(const orc_mw_game* g, const orc_mw_ctx* c, int i, int sem,
                            const float* const* reach /* [4] at node i */, float* out /* [4][H] */) {
    const mtt_mw_node* nd = &g->nodes[i];
    int H = g->H;
    int am = nd->active_mask;
    if (sem == ORC_SEM_REFERENCE) {
        double tot[4];
        double* cdf[4];
        for (int o = 0; o < 4; ++o) {
            cdf[o] = (double*)calloc((size_t)H + 1, sizeof(double));
            double* byp = (double*)calloc((size_t)H + 1, sizeof(double));
            for (int h = 0; h < H; ++h) byp[c->pos[h]] = reach[o][h];
            double run = 0.0;
            for (int k = 0; k < H; ++k) { cdf[o][k] = run; run += byp[k]; }
            cdf[o][H] = run;
            tot[o] = run;
            free(byp);
        }
        for (int p = 0; p < 4; ++p) {
            double others = 1.0;
            for (int o = 0; o < 4; ++o) if (o != p) others *= tot[o];
            for (int h = 0; h < H; ++h) {
                double v;
                if (nd->type == MTT_NODE_FOLD) {
                    int w = 0;
                    while (!((am >> w) & 1)) ++w;
                    v = (p == w ? (double)nd->pot_size - (double)nd->committed[p]
                                : -(double)g->bubble[p * 4 + w] * (double)nd->committed[p]) * others;
                } else if (!((am >> p) & 1)) {
                    v = -(double)g->bubble[p * 4 + p] * (double)nd->committed[p] * others;
                } else {
                    double gain = (double)nd->pot_size - (double)nd->committed[p];
                    double loss = -(double)g->bubble[p * 4 + p] * (double)nd->committed[p];
                    double inact = 1.0, PW = 1.0, F = 1.0;
                    for (int o = 0; o < 4; ++o) {
                        if (o == p) continue;
                        if ((am >> o) & 1) { PW *= tot[o]; F *= cdf[o][c->pos[h]]; } else inact *= tot[o];
                    }
                    v = (gain * F + loss * (PW - F)) * inact;
                }
                out[(size_t)p * H + h] = (float)v;
            }
        }
        for (int o = 0; o < 4; ++o) free(cdf[o]);
        return;
    }
    /* correct semantics: per hero hand h and opponent o, the masses of o's
     * hands that share no card with h */
    double* L = (double*)malloc(sizeof(double) * 4 * (size_t)H);
    double* E = (double*)malloc(sizeof(double) * 4 * (size_t)H);
    double* W = (double*)malloc(sizeof(double) * 4 * (size_t)H);
    #pragma omp parallel for schedule(static)
    for (int h = 0; h < H; ++h) {
        for (int o = 0; o < 4; ++o) {
            double l = 0.0, e = 0.0, w = 0.0;
            for (int j = 0; j < H; ++j) {
                if (c->mask[j] & c->mask[h]) continue;
                double r = (double)reach[o][j];
                w += r;
                if (c->sc[j] < c->sc[h]) l += r;
                else if (c->sc[j] == c->sc[h]) e += r;
            }
            L[(size_t)o * H + h] = l; E[(size_t)o * H + h] = e; W[(size_t)o * H + h] = w;
        }
    }
    for (int p = 0; p < 4; ++p) {
        for (int h = 0; h < H; ++h) {
            double others = 1.0;
            for (int o = 0; o < 4; ++o) if (o != p) others *= W[(size_t)o * H + h];
            double v;
            if (nd->type == MTT_NODE_FOLD) {
                int w = 0;
                while (!((am >> w) & 1)) ++w;
                v = (p == w ? (double)nd->pot_size - (double)nd->committed[p]
                            : -(double)g->bubble[p * 4 + w] * (double)nd->committed[p]) * others;
            } else if (!((am >> p) & 1)) {
                v = -(double)g->bubble[p * 4 + p] * (double)nd->committed[p] * others;
            } else {
                double loss = -(double)g->bubble[p * 4 + p] * (double)nd->committed[p];
                double inact = 1.0, PW = 1.0, LE = 1.0, share = 0.0;
                double Lk[3], Ek[3];
                int no = 0;
                for (int o = 0; o < 4; ++o) {
                    if (o == p) continue;
                    if ((am >> o) & 1) {
                        Lk[no] = L[(size_t)o * H + h];
                        Ek[no] = E[(size_t)o * H + h];
                        PW *= W[(size_t)o * H + h];
                        LE *= Lk[no] + Ek[no];
                        ++no;
                    } else {
                        inact *= W[(size_t)o * H + h];
                    }
                }
                for (int T = 0; T < (1 << no); ++T) {
                    double pr = 1.0;
                    int nt = 0;
                    for (int k = 0; k < no; ++k) {
                        if ((T >> k) & 1) { pr *= Ek[k]; ++nt; } else pr *= Lk[k];
                    }
                    share += pr * ((double)nd->pot_size / (1 + nt) - (double)nd->committed[p]);
                }
                v = (share + loss * (PW - LE)) * inact;
            }
            out[(size_t)p * H + h] = (float)v;
        }
    }
    free(L); free(E); free(W);
}

/* One terminal's values under the solver's semantics (the routine the sweep
 * below calls), for tests: out [4][H]. */
int orc_mw_terminal_values(const orc_mw_game* g, int i, int sem, const float* const* reach, float* out) {
    if (!g || g->H < 1 || i < 0 || i >= g->n_nodes) return MTT_ERR_INVALID;
    orc_mw_ctx c;
    orc_mw_ranks(g, &c);
    orc_mw_terminal(g, &c, i, sem, reach, out);
    orc_mw_free(&c);
    return MTT_OK;
}

/* The exact four-player showdown of the hand (no approximation): player p's
 * value of hand h, summed over every assignment of hands to the other three
 * players in which all four hands are disjoint, each weighted by the product
 * of the three reaches; fold and inactive payoffs as above, equal hands split
 * the pot among the active players holding them.  O(H^3) per hand: small
 * cases only (a check of how far the hero-conditioned masses above are from
 * the exact game). */
int orc_mw_exact_terminal(const orc_mw_game* g, int i, const float* const* reach, double* out) {
    if (!g || g->H < 1 || i < 0 || i >= g->n_nodes) return MTT_ERR_INVALID;
    orc_mw_ctx c;
    orc_mw_ranks(g, &c);
    const mtt_mw_node* nd = &g->nodes[i];
    int H = g->H, am = nd->active_mask;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int h = 0; h < H; ++h) {
        for (int p = 0; p < 4; ++p) {
            int opp[3], no = 0;
            for (int o = 0; o < 4; ++o) if (o != p) opp[no++] = o;
            double acc = 0.0;
            for (int j0 = 0; j0 < H; ++j0) {
                if (c.mask[j0] & c.mask[h]) continue;
                double r0 = (double)reach[opp[0]][j0];
                if (r0 == 0.0) continue;
                uint64_t m0 = c.mask[h] | c.mask[j0];
                for (int j1 = 0; j1 < H; ++j1) {
                    if (c.mask[j1] & m0) continue;
                    double r1 = r0 * (double)reach[opp[1]][j1];
                    if (r1 == 0.0) continue;
                    uint64_t m1 = m0 | c.mask[j1];
                    for (int j2 = 0; j2 < H; ++j2) {
                        if (c.mask[j2] & m1) continue;
                        double w = r1 * (double)reach[opp[2]][j2];
                        if (w == 0.0) continue;
                        double u;
                        if (nd->type == MTT_NODE_FOLD) {
                            int win = 0;
                            while (!((am >> win) & 1)) ++win;
                            u = p == win ? (double)nd->pot_size - (double)nd->committed[p]
                                         : -(double)g->bubble[p * 4 + win] * (double)nd->committed[p];
                        } else if (!((am >> p) & 1)) {
                            u = -(double)g->bubble[p * 4 + p] * (double)nd->committed[p];
                        } else {
                            int js[3] = {j0, j1, j2}, beaten = 0, ties = 0;
                            for (int k = 0; k < 3; ++k) {
                                if (!((am >> opp[k]) & 1)) continue;
                                if (c.sc[js[k]] > c.sc[h]) beaten = 1;
                                else if (c.sc[js[k]] == c.sc[h]) ++ties;
                            }
                            u = beaten ? -(double)g->bubble[p * 4 + p] * (double)nd->committed[p]
                                       : (double)nd->pot_size / (1 + ties) - (double)nd->committed[p];
                        }
                        acc += w * u;
                    }
                }
            }
            out[(size_t)p * H + h] = acc;
        }
    }
    orc_mw_free(&c);
    return MTT_OK;
}

static float orc_mw_sigma(const float* B, int H, int A, int k, int h, int avg) {
    float sum = 0.0f;
    for (int j = 0; j < A; ++j) sum += avg ? B[(size_t)j * H + h] : fmaxf(B[(size_t)j * H + h], 0.0f);
    float invA = 1.0f / (float)A;
    if (avg) return sum > 0.0f ? B[(size_t)k * H + h] / sum : invA;
    return sum > 1e-7f ? fmaxf(B[(size_t)k * H + h], 0.0f) / sum : invA;
}

/* One sweep: reach down, terminals, values up; updates when upd != 0. */
static void orc_mw_sweep(const orc_mw_game* g, const orc_mw_ctx* c, const orc_cfr_params* prm, int t,
                         float** R, float** S, float* reach, float* cfv, int upd, int sem) {
    int n = g->n_nodes, H = g->H;
    size_t HS = (size_t)4 * H;
    for (int p = 0; p < 4; ++p) for (int h = 0; h < H; ++h) reach[(size_t)p * H + h] = g->range[p][h];
    for (int i = 0; i < n; ++i) {
        const mtt_mw_node* nd = &g->nodes[i];
        if (nd->type != MTT_NODE_DECISION) continue;
        int p = nd->player, A = nd->num_actions;
        const float* B = (upd ? R[p] : S[p]) + (size_t)nd->infoset_offset * H;
        for (int a = 0; a < A; ++a) {
            int ch = nd->children_offset + a;
            memcpy(&reach[(size_t)ch * HS], &reach[(size_t)i * HS], sizeof(float) * HS);
            for (int h = 0; h < H; ++h)
                reach[(size_t)ch * HS + (size_t)p * H + h] = reach[(size_t)i * HS + (size_t)p * H + h] *
                                                             orc_mw_sigma(B, H, A, a, h, !upd);
        }
    }
    double tm1 = (double)(t - 1);
    float w_lin = (float)pow((double)t, (double)prm->avg_power);
    float dpos = (float)(pow(tm1, (double)prm->alpha) / (pow(tm1, (double)prm->alpha) + 1.0));
    float dneg = (float)(pow(tm1, (double)prm->beta) / (pow(tm1, (double)prm->beta) + 1.0));
    float dstr = (float)pow(tm1 / (double)t, (double)prm->gamma);
    for (int i = n - 1; i >= 0; --i) {
        const mtt_mw_node* nd = &g->nodes[i];
        float* out = &cfv[(size_t)i * HS];
        if (nd->type != MTT_NODE_DECISION) {
            const float* rp[4];
            for (int p = 0; p < 4; ++p) rp[p] = &reach[(size_t)i * HS + (size_t)p * H];
            orc_mw_terminal(g, c, i, sem, rp, out);
            continue;
        }
        int p = nd->player, A = nd->num_actions;
        for (int q = 0; q < 4; ++q) {
            for (int h = 0; h < H; ++h) {
                if (q != p) {
                    float s = 0.0f;
                    for (int a = 0; a < A; ++a) s += cfv[(size_t)(nd->children_offset + a) * HS + (size_t)q * H + h];
                    out[(size_t)q * H + h] = s;
                }
            }
        }
        float* Rb = R[p] + (size_t)nd->infoset_offset * H;
        float* Sb = S[p] + (size_t)nd->infoset_offset * H;
        const float* B = upd ? Rb : Sb;
        for (int h = 0; h < H; ++h) {
            float sg[MTT_MW_MAX_ACTIONS], v = 0.0f;
            for (int a = 0; a < A; ++a) {
                sg[a] = orc_mw_sigma(B, H, A, a, h, !upd);
                v = fmaf(sg[a], cfv[(size_t)(nd->children_offset + a) * HS + (size_t)p * H + h], v);
            }
            out[(size_t)p * H + h] = v;
            if (!upd) continue;
            float r = reach[(size_t)i * HS + (size_t)p * H + h];
            float wr = r * w_lin;
            for (int a = 0; a < A; ++a) {
                float qk = cfv[(size_t)(nd->children_offset + a) * HS + (size_t)p * H + h];
                float rk = Rb[(size_t)a * H + h], inst = qk - v;
                float sv = Sb[(size_t)a * H + h];
                if (prm->algo == ORC_ALGO_DCFR) {
                    Rb[(size_t)a * H + h] = rk * (rk > 0.0f ? dpos : dneg) + inst;
                    Sb[(size_t)a * H + h] = fmaf(r, sg[a], sv * dstr);
                } else {
                    Rb[(size_t)a * H + h] = fmaxf(0.0f, rk + inst);
                    Sb[(size_t)a * H + h] = fmaf(wr, sg[a], sv);
                }
            }
        }
    }
}

int orc_mw_solve(const orc_mw_game* g, const orc_cfr_params* prm, float* R[4], float* S[4], float* root_cfv,
                 double* values) {
    if (!g || !prm || g->H < 1) return MTT_ERR_INVALID;
    orc_mw_ctx c;
    orc_mw_ranks(g, &c);
    int n = g->n_nodes, H = g->H;
    size_t HS = (size_t)4 * H;
    float* reach = (float*)calloc((size_t)n * HS + 1, sizeof(float));
    float* cfv = (float*)calloc((size_t)n * HS + 1, sizeof(float));
    for (int p = 0; p < 4; ++p) {
        memset(R[p], 0, sizeof(float) * (size_t)g->rows[p] * (size_t)H);
        memset(S[p], 0, sizeof(float) * (size_t)g->rows[p] * (size_t)H);
    }
    for (int t = 1; t <= prm->iters; ++t) orc_mw_sweep(g, &c, prm, t, R, S, reach, cfv, 1, prm->semantics);
    if (root_cfv) memcpy(root_cfv, cfv, sizeof(float) * HS);
    if (values) {
        orc_mw_sweep(g, &c, prm, 1, R, S, reach, cfv, 0, prm->semantics);
        for (int p = 0; p < 4; ++p) {
            double acc = 0.0;
            for (int h = 0; h < H; ++h) acc += (double)g->range[p][h] * (double)cfv[(size_t)p * H + h];
            values[p] = acc;
        }
    }
    free(reach); free(cfv); orc_mw_free(&c);
    return MTT_OK;
}

/* Malmuth-Harville equity by direct enumeration of the ordered finishers of
 * the paid places (an independent restatement of the subset recursion). */
static void orc_icm_rec(const double* st, int n, const double* pay, int m, int depth, unsigned used, double rest,
                        double prob, double* out) {
    if (depth == m || !(rest > 0.0)) return;
    for (int i = 0; i < n; ++i) {
        if ((used >> i) & 1u) continue;
        double p = prob * st[i] / rest;
        if (p == 0.0) continue;
        out[i] += p * pay[depth];
        orc_icm_rec(st, n, pay, m, depth + 1, used | (1u << i), rest - st[i], p, out);
    }
}

int orc_icm_equity(const double* stacks, int n, const double* payouts, int m, double* out) {
    if (n < 1 || n > 16 || m < 0 || m > n) return MTT_ERR_INVALID;
    double S = 0.0;
    for (int i = 0; i < n; ++i) { out[i] = 0.0; S += stacks[i]; }
    orc_icm_rec(stacks, n, payouts, m, 0, 0u, S, 1.0, out);
    return MTT_OK;
}

/* ------------------------------------------------------------------------ */
/* Preflop anchor chain: restates src/preflop/preflop_grid_generator.cu      */
/* (kernels :95-421, host set-up and loop :426-614) in reference mode.       */
/* ------------------------------------------------------------------------ */
#define PF_CLASSES 169
#define PF_PAD 192
#define PF_ALIVE 1176
#define PF_PADDED 1216

/* class_to_cards (:79-92), including its boundary behaviour: the last class
 * of each rank group maps to the next group (e.g. A2s to two copies of the
 * king of clubs).  For the last suited and the last offsuit class (90, 168)
 * the reference's loop never leaves through its condition (it runs into
 * signed overflow, undefined behaviour); there the class's own cards
 * (3c2c, 3c2d) are used. */
static void orc_pf_class_to_cards(int cls, uint8_t* h1, uint8_t* h2) {
    if (cls < 13) { int r = 12 - cls; *h1 = (uint8_t)(r * 4 + 0); *h2 = (uint8_t)(r * 4 + 1); }
    else {
        int base = cls < 91 ? 13 : 91, r1 = 12, r2;
        while (r1 > 0 && base + (r1 - 1) <= cls) base += r1--;
        if (r1 == 0) { *h1 = 4; *h2 = (uint8_t)(cls < 91 ? 0 : 1); return; }
        r2 = r1 - 1 - (cls - base);
        *h1 = (uint8_t)(r1 * 4 + 0);
        *h2 = (uint8_t)(r2 * 4 + (cls < 91 ? 0 : 1));
    }
}

/* combo -> class as the host set-up computes it (:475-483) */
int orc_pf_combo_class(int c1, int c2) {
    int r1 = c1 / 4, s1 = c1 % 4, r2 = c2 / 4, s2 = c2 % 4;
    int hi = r1 > r2 ? r1 : r2, lo = r1 < r2 ? r1 : r2;
    if (r1 == r2) return 12 - hi;
    int base = (s1 == s2) ? 13 : 91;
    for (int r = 12; r > hi; --r) base += r;
    return base + (hi - 1 - lo);
}

/* kernel_gen_preflop_matrix (:95-127): 3,000 LCG board samples per class pair */
void orc_pf_allin_matrix(int hc_begin, int hc_end, float* out, int32_t* wins_out, int32_t* ties_out) {
    #pragma omp parallel for schedule(dynamic, 1)
    for (int hc = hc_begin; hc < hc_end; ++hc)
        for (int vc = 0; vc < PF_CLASSES; ++vc) {
            float* o = &out[hc * PF_CLASSES + vc];
            if (wins_out) { wins_out[hc * PF_CLASSES + vc] = 0; ties_out[hc * PF_CLASSES + vc] = 0; }
            if (hc == vc) { *o = 0.5f; continue; }
            uint8_t h1, h2, v1, v2;
            orc_pf_class_to_cards(hc, &h1, &h2);
            orc_pf_class_to_cards(vc, &v1, &v2);
            if (h1 == v1 || h1 == v2 || h2 == v1 || h2 == v2) {
                if (h1 == v1 || h2 == v1) v1 = (uint8_t)((v1 / 4) * 4 + 2);
                if (h1 == v2 || h2 == v2) v2 = (uint8_t)((v2 / 4) * 4 + 3);
            }
            uint64_t dead = (1ull << h1) | (1ull << h2) | (1ull << v1) | (1ull << v2);
            uint8_t deck[52]; int dsz = 0;
            for (int c = 0; c < 52; ++c) if (!(dead & (1ull << c))) deck[dsz++] = (uint8_t)c;
            uint32_t rng = (uint32_t)(hc * 169 + vc) * 2654435761u + 0x9E3779B9u;
            int wins = 0, ties = 0;
            uint8_t a[7] = {h1, h2, 0, 0, 0, 0, 0}, b[7] = {v1, v2, 0, 0, 0, 0, 0};
            for (int s = 0; s < 3000; ++s) {
                uint8_t bd[5];
                for (int k = 0; k < 5; ++k) {
                    rng = rng * 1664525u + 1013904223u;
                    int pick = k + (int)((rng >> 16) % (uint32_t)(dsz - k));
                    bd[k] = deck[pick];
                }
                for (int k = 0; k < 5; ++k) { a[2 + k] = bd[k]; b[2 + k] = bd[k]; }
                uint32_t sh = orc_score7(a), sv = orc_score7(b);
                if (sh > sv) wins++; else if (sh == sv) ties++;
            }
            *o = ((float)wins + 0.5f * (float)ties) / 3000.0f;
            if (wins_out) { wins_out[hc * PF_CLASSES + vc] = wins; ties_out[hc * PF_CLASSES + vc] = ties; }
        }
}

/* The alive-combo list and per-class lists of the host set-up (:467-495):
 * the first 1,176 combos in lexicographic order, at most 12 per class. */
static void orc_pf_lists(uint8_t* cc /* [1176][2] */, int* cls_count /* [169] */, int* cls_idx /* [169][12] */) {
    int n = 0;
    for (int k = 0; k < PF_CLASSES; ++k) cls_count[k] = 0;
    for (int c1 = 0; c1 < 52; ++c1)
        for (int c2 = c1 + 1; c2 < 52; ++c2) {
            if (n >= PF_ALIVE) continue;
            int cls = orc_pf_combo_class(c1, c2);
            cc[2 * n] = (uint8_t)c1; cc[2 * n + 1] = (uint8_t)c2;
            if (cls_count[cls] < 12) cls_idx[cls * 12 + cls_count[cls]++] = n;
            ++n;
        }
}

/* kernel_gen_100_flop_matrices (:130-183) for one flop, then
 * kernel_reduce_combo_to_class_matrices (:189-223).  Entries of hero combos
 * that touch the flop are never written by the reference (its buffer is
 * uninitialised); here they read as 0, which the reduction skips (eq > 0).
 * out_class[v_cls * 169 + h_cls]. */
void orc_pf_flop_class_matrix(const uint8_t flop[3], float* out_class, float* out_combo /* optional [1216*1216] */) {
    uint8_t cc[2 * PF_ALIVE];
    int cnt[PF_CLASSES], idx[PF_CLASSES * 12];
    orc_pf_lists(cc, cnt, idx);
    float* E = out_combo ? out_combo : (float*)malloc(sizeof(float) * PF_PADDED * PF_PADDED);
    memset(E, 0, sizeof(float) * PF_PADDED * PF_PADDED);
    uint64_t fm = (1ull << flop[0]) | (1ull << flop[1]) | (1ull << flop[2]);
    #pragma omp parallel for schedule(dynamic, 8)
    for (int h = 0; h < PF_ALIVE; ++h) {
        uint64_t hm = (1ull << cc[2 * h]) | (1ull << cc[2 * h + 1]);
        if (hm & fm) continue;
        uint64_t dhf = hm | fm;
        uint8_t deck[52]; int dsz = 0;
        for (int c = 0; c < 52; ++c) if (!(dhf & (1ull << c))) deck[dsz++] = (uint8_t)c;
        for (int j = 0; j < PF_ALIVE; ++j) {
            uint64_t vm = (1ull << cc[2 * j]) | (1ull << cc[2 * j + 1]);
            if ((hm & vm) || (vm & fm)) { E[(size_t)j * PF_PADDED + h] = 0.0f; continue; }
            uint8_t a[7] = {flop[0], flop[1], flop[2], cc[2 * h], cc[2 * h + 1], 0, 0};
            uint8_t b[7] = {flop[0], flop[1], flop[2], cc[2 * j], cc[2 * j + 1], 0, 0};
            uint64_t dall = dhf | vm;
            int wins = 0, ties = 0, total = 0;
            for (int r1 = 0; r1 < dsz; r1 += 2) {
                uint8_t t = deck[r1];
                if (dall & (1ull << t)) continue;
                a[5] = t; b[5] = t;
                for (int r2 = r1 + 1; r2 < dsz; r2 += 3) {
                    uint8_t r = deck[r2];
                    if (dall & (1ull << r)) continue;
                    a[6] = r; b[6] = r;
                    uint32_t sh = orc_score7(a), sv = orc_score7(b);
                    if (sh > sv) wins += 2; else if (sh == sv) ties += 1;
                    total += 2;
                }
            }
            E[(size_t)j * PF_PADDED + h] = total > 0 ? ((float)wins + 0.5f * (float)ties) / (float)total : 0.0f;
        }
    }
    for (int hc = 0; hc < PF_CLASSES; ++hc)
        for (int vc = 0; vc < PF_CLASSES; ++vc) {
            float sum = 0.0f;
            int valid = 0;
            for (int i = 0; i < cnt[hc]; ++i)
                for (int j = 0; j < cnt[vc]; ++j) {
                    float eq = E[(size_t)idx[vc * 12 + j] * PF_PADDED + idx[hc * 12 + i]];
                    if (eq > 0.0f) { sum += eq; valid++; }
                }
            out_class[vc * PF_CLASSES + hc] = valid > 0 ? sum / (float)valid : 0.5f;
        }
    if (!out_combo) free(E);
}

/* The closed preflop tree and DCFR loop (:224-421, :563-614): BTN root
 * (fold / min-raise / jam), BB vs min-raise (fold / call / 3-bet jam), BTN vs
 * 3-bet jam (fold / call), BB vs open jam (fold / call); flop play is the
 * co-solve over the class-reduced board matrices.  class_mats: [n][v][h]. */

static void orc_pf_cosolve(int nf, const float* fw, const float* rbc, const float* rbb, const float* mats,
                           float* ev_btn, float* ev_bb, float pot_flop, float bf) {
    for (int cls = 0; cls < PF_CLASSES; ++cls) {
        float acc_btn = 0.0f, acc_bb = 0.0f, tw = 0.0f;
        for (int f = 0; f < nf; ++f) {
            float w = fw[f];
            tw += w;
            const float* eq = &mats[(size_t)f * PF_CLASSES * PF_CLASSES];
            float s1 = 0.0f, e0 = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) { float r = rbb[o]; s1 += r; e0 += r * eq[o * PF_CLASSES + cls]; }
            if (s1 > 1e-7f) e0 /= s1;
            float s0 = 0.0f, e1 = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) { float r = rbc[o]; s0 += r; e1 += r * (1.0f - eq[cls * PF_CLASSES + o]); }
            if (s0 > 1e-7f) e1 /= s0;
            float sh_btn = e0 * 1.06f * pot_flop, sh_bb = e1 * 0.94f * pot_flop;
            float nb = sh_btn >= 2.1f ? sh_btn - 2.1f : -((2.1f - sh_btn) * bf);
            float nbb = sh_bb >= 2.1f ? sh_bb - 2.1f : -((2.1f - sh_bb) * bf);
            acc_btn += w * nb;
            acc_bb += w * nbb;
        }
        if (tw > 0.0f) { ev_btn[cls] = acc_btn / tw; ev_bb[cls] = acc_bb / tw; }
    }
}

static void orc_pf_dcfr_step(int A, float* R, float* sig, float* S, const float* cfv, const float* reach, float wp, float ws) {
    for (int cls = 0; cls < PF_CLASSES; ++cls) {
        float v = 0.0f;
        for (int a = 0; a < A; ++a) v += sig[a * PF_PAD + cls] * cfv[a * PF_PAD + cls];
        float pos = 0.0f, nxt[3] = {0.0f, 0.0f, 0.0f};
        for (int a = 0; a < A; ++a) {
            int i = a * PF_PAD + cls;
            float nr = wp * fmaxf(0.0f, R[i] + (cfv[i] - v));
            R[i] = nr; pos += nr; nxt[a] = nr;
            S[i] += ws * reach[cls] * sig[i];
        }
        for (int a = 0; a < A; ++a) sig[a * PF_PAD + cls] = pos > 1e-7f ? nxt[a] / pos : 1.0f / (float)A;
    }
}

/* sums: 4 blocks [3|3|2|2][192] (BTN root, BB defence, BTN vs 3-bet, BB vs jam). */
int orc_pf_dcfr(int nf, const float* flop_weights, const float* class_mats, const float* allin,
                const orc_pf_params* p, float* sums, float* sigma) {
    const int A[4] = {3, 3, 2, 2};
    float *R[4], *G[4], *S[4], *C[4];
    for (int k = 0; k < 4; ++k) {
        R[k] = (float*)calloc((size_t)A[k] * PF_PAD, sizeof(float));
        G[k] = (float*)calloc((size_t)A[k] * PF_PAD, sizeof(float));
        S[k] = (float*)calloc((size_t)A[k] * PF_PAD, sizeof(float));
        C[k] = (float*)calloc((size_t)A[k] * PF_PAD, sizeof(float));
        for (int i = 0; i < A[k] * PF_PAD; ++i) G[k][i] = 1.0f / (float)A[k];
    }
    float root[PF_PAD] = {0}, rbc[PF_PAD] = {0}, rbb[PF_PAD] = {0}, evb[PF_PAD] = {0}, evbb[PF_PAD] = {0};
    for (int c = 0; c < PF_CLASSES; ++c) root[c] = (c < 13 ? 6.0f : c < 91 ? 4.0f : 12.0f) / 1326.0f;
    const float dead = p->dead_pot, stack = p->stack_bb, bf = p->bubble;
    const float jam_pot = 2.0f * stack + dead;
    for (int t = 1; t <= p->iters; ++t) {
        float tf = (float)t;
        float wp = powf(tf, 1.5f) / (powf(tf, 1.5f) + 1.0f), ws = tf * tf;
        for (int c = 0; c < PF_CLASSES; ++c) {            /* kernel_update_dynamic_reaches */
            rbc[c] = root[c] * G[0][1 * PF_PAD + c];
            rbb[c] = root[c] * G[1][1 * PF_PAD + c];
        }
        orc_pf_cosolve(nf, flop_weights, rbc, rbb, class_mats, evb, evbb, dead + 3.1f, bf);
        for (int cls = 0; cls < PF_CLASSES; ++cls) {       /* kernel_build_closed_preflop_cfvs */
            const float *sbr = G[0], *sbd = G[1], *s3b = G[2], *sbj = G[3];
            C[2][0 * PF_PAD + cls] = -2.1f * bf;
            float m3 = 0.0f, eqc = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) { float r = root[o] * sbd[2 * PF_PAD + o]; m3 += r; eqc += r * allin[cls * PF_CLASSES + o]; }
            if (m3 > 1e-7f) eqc /= m3;
            C[2][1 * PF_PAD + cls] = eqc * (jam_pot - stack) - (1.0f - eqc) * bf * stack;
            float v3 = s3b[0 * PF_PAD + cls] * C[2][0 * PF_PAD + cls] + s3b[1 * PF_PAD + cls] * C[2][1 * PF_PAD + cls];
            C[1][0 * PF_PAD + cls] = -1.0f * bf;
            C[1][1 * PF_PAD + cls] = evbb[cls];
            float bf3 = 0.0f, bc3 = 0.0f, eqj = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) {
                float ro = root[o] * sbr[1 * PF_PAD + o];
                bf3 += ro * s3b[0 * PF_PAD + o];
                bc3 += ro * s3b[1 * PF_PAD + o];
                eqj += ro * s3b[1 * PF_PAD + o] * (1.0f - allin[o * PF_CLASSES + cls]);
            }
            if (bc3 > 1e-7f) eqj /= bc3;
            float tot3 = bf3 + bc3 + 1e-9f;
            float evsh = eqj * (jam_pot - stack) - (1.0f - eqj) * bf * stack;
            C[1][2 * PF_PAD + cls] = (bf3 * (dead + 2.1f) + bc3 * evsh) / tot3;
            C[3][0 * PF_PAD + cls] = -1.0f * bf;
            float mj = 0.0f, eqo = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) { float r = root[o] * sbr[2 * PF_PAD + o]; mj += r; eqo += r * (1.0f - allin[o * PF_CLASSES + cls]); }
            if (mj > 1e-7f) eqo /= mj;
            C[3][1 * PF_PAD + cls] = eqo * (jam_pot - stack) - (1.0f - eqo) * bf * stack;
            C[0][0 * PF_PAD + cls] = 0.0f;
            float fm = 0.0f, cm = 0.0f, jm = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) {
                float r = root[o];
                fm += r * sbd[0 * PF_PAD + o]; cm += r * sbd[1 * PF_PAD + o]; jm += r * sbd[2 * PF_PAD + o];
            }
            float tb = fm + cm + jm + 1e-9f;
            C[0][1 * PF_PAD + cls] = (fm * dead + cm * evb[cls] + jm * v3) / tb;
            float fj = 0.0f, cj = 0.0f, eo = 0.0f;
            for (int o = 0; o < PF_CLASSES; ++o) {
                float r = root[o];
                fj += r * sbj[0 * PF_PAD + o]; cj += r * sbj[1 * PF_PAD + o];
                eo += r * sbj[1 * PF_PAD + o] * allin[cls * PF_CLASSES + o];
            }
            float toj = fj + cj + 1e-9f;
            if (cj > 1e-7f) eo /= cj;
            C[0][2 * PF_PAD + cls] = (fj * dead + cj * (eo * (jam_pot - stack) - (1.0f - eo) * bf * stack)) / toj;
        }
        orc_pf_dcfr_step(3, R[0], G[0], S[0], C[0], root, wp, ws);
        orc_pf_dcfr_step(3, R[1], G[1], S[1], C[1], root, wp, ws);
        orc_pf_dcfr_step(2, R[2], G[2], S[2], C[2], root, wp, ws);
        orc_pf_dcfr_step(2, R[3], G[3], S[3], C[3], root, wp, ws);
    }
    size_t o = 0;
    for (int k = 0; k < 4; ++k) {
        if (sums) memcpy(sums + o, S[k], sizeof(float) * (size_t)A[k] * PF_PAD);
        if (sigma) memcpy(sigma + o, G[k], sizeof(float) * (size_t)A[k] * PF_PAD);
        o += (size_t)A[k] * PF_PAD;
        free(R[k]); free(G[k]); free(S[k]); free(C[k]);
    }
    return MTT_OK;
}
