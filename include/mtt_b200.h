/*
 * mtt_b200.h — C ABI of the B200 (sm_100a) hot path of MTT-GPU-Solver.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (MTT_OK == 0) and never exits the process.  Unless stated otherwise,
 * pointers whose name starts with d_ are device pointers owned by the caller,
 * h_ pointers are host pointers, and `stream` is a cudaStream_t passed as
 * void* (NULL = the legacy default stream).  Calls on different devices or
 * different streams may run concurrently from different host threads; a
 * handle (mtt_solver / mtt_batch) is used by one host thread at a time.
 *
 * Card encoding follows the reference: card = rank*4 + suit, rank 0='2' ..
 * 12='A', suit 0..3 = c,d,h,s (src/tools/mtt_ev_dumper.cu:27,
 * scripts/optimize_subset.py:59-61).  A hole-card combo is an unordered pair
 * (c1 < c2); combo ids 0..1325 enumerate the pairs lexicographically.
 *
 * Reference citations are file:line inside the MTT-GPU-Solver project.
 */
#ifndef MTT_B200_H
#define MTT_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; everything declared here is exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ------------------------------------------------------------------ status */
#define MTT_OK              0
#define MTT_ERR_INVALID     1   /* bad argument, size or tree */
#define MTT_ERR_CUDA        2   /* a CUDA runtime call failed (see mtt_last_cuda_error) */
#define MTT_ERR_NOMEM       3   /* device or host allocation failed */
#define MTT_ERR_TIMEOUT     4   /* a bounded device wait gave up */
#define MTT_ERR_IO          5   /* file missing, short or malformed */
#define MTT_ERR_UNSUPPORTED 6   /* size or feature outside what this build handles */

/* Human-readable name of a status code (static string). */
const char* mtt_status_string(int status);
/* cudaError_t value of the last failing CUDA call on this host thread (0 if none). */
int mtt_last_cuda_error(void);
/* Library version string. */
const char* mtt_version(void);
/* Self-check of the bounded device waits (no reference counterpart).  One
 * CTA waits on an mbarrier that no copy targets, giving up after limit_us
 * microseconds (1 .. 2,000,000).  arrive = 0: nothing arrives, the wait runs
 * out and the call returns MTT_ERR_TIMEOUT, the status every kernel with a
 * bounded wait reports when it gives up; arrive != 0: one thread arrives
 * first and the call returns MTT_OK.  No copy is left in flight either way,
 * so the device stays usable.  Synchronous. */
int mtt_selftest_bounded_wait(int32_t arrive, int32_t limit_us, void* stream);

/* ------------------------------------------------------------- game trees */
#define MTT_NODE_DECISION 0
#define MTT_NODE_FOLD     1
#define MTT_NODE_SHOWDOWN 2
#define MTT_NODE_CHANCE   3
/* Depth-limit leaf (no reference counterpart): the turn betting round closed
 * with chips behind; the river that follows is valued by a leaf network
 * (mtt_batch_set_leafnet).  reserved = the chips each player has behind. */
#define MTT_NODE_LEAF     4

/* Flat heads-up tree node, 32 bytes.  The field order, widths and meaning
 * follow the reference's FlatNode (src/postflop/honest_multistreet_solver.cu:14-21):
 * children are contiguous at children_offset + a; a fold node's active_mask
 * has the bit of the player who did NOT fold; pot_size and committed[] are
 * chips, and each player's committed[] includes half of the starting pot, so
 * payoffs are zero-sum.  Two differences, both in fields the reference leaves
 * implicit: infoset_offset is the first row of this node in ITS PLAYER's own
 * regret array (rows are numbered per player, one row per action, so the
 * reference's info*MAX_ACTIONS+a becomes infoset_offset+a), and the 2-byte
 * pad after turn_idx holds the node depth.  turn_idx is the card dealt by the
 * parent chance node (-1 when there is none). */
typedef struct mtt_node {
    uint8_t  type;
    uint8_t  player;
    uint8_t  num_actions;
    uint8_t  active_mask;
    int32_t  children_offset;
    int32_t  infoset_offset;
    int16_t  turn_idx;
    int16_t  depth;
    float    pot_size;
    float    committed[2];
    float    reserved;
} mtt_node;

#define MTT_MAX_SIZES 8
/* Betting abstraction for one heads-up subgame.  Sizes are fractions of the
 * pot; a raise size f puts in to_call + f*(pot + to_call).  Any size at or
 * above the remaining stack becomes all-in.  raise_cap counts raises after
 * the first bet of a street. street = 5: river subgame (5-card board);
 * street = 4: turn subgame whose betting rounds close into a river chance
 * node (48 children) followed by a river subgame with the same sizes;
 * street = 3: flop subgame (the reference's multistreet structure,
 * honest_multistreet_solver.cu:97-104,205-219): flop betting, a turn chance
 * node (49 children), turn betting, then the river dealt (48 children) to
 * showdowns without river betting. */
typedef struct mtt_tree_spec {
    float   pot;
    float   stack;
    int32_t n_bet_sizes;
    float   bet_sizes[MTT_MAX_SIZES];
    int32_t n_raise_sizes;              /* 0: raises reuse bet_sizes */
    float   raise_sizes[MTT_MAX_SIZES];
    int32_t raise_cap;
    int32_t allin;                      /* 1: all-in is always offered */
    int32_t street;                     /* 5, 4 or 3 */
    int32_t river_leaves;               /* street 4: rounds that close with chips behind end in
                                           MTT_NODE_LEAF instead of a river chance node */
    int32_t river_runout;               /* street 4: the river is dealt straight to showdowns
                                           (no river betting); always so for street 3 */
} mtt_tree_spec;

/* Build the tree in breadth-first order (children contiguous, parents first).
 * nodes may be NULL to query the size.  Outputs: *n_nodes, rows per player
 * (rows[2]: regret rows of player 0 and 1), *max_depth. Host only. */
int mtt_tree_build(const mtt_tree_spec* spec, mtt_node* nodes, int32_t capacity,
                   int32_t* n_nodes, int32_t rows[2], int32_t* max_depth);

/* Turn subgame (spec->street == 4, board = 4 cards): every betting round that
 * closes with chips behind goes to a river chance node with one child per
 * card not on the board, followed by a river round (showdowns with
 * river_runout); all-in calls go to a chance node whose children are
 * showdowns.  Flop subgame (street == 3, board = 3 cards): the same one street
 * earlier, with a turn chance node (one child per card not on the board)
 * before the turn round and the river run out; an all-in deals the turn and
 * then the river.  Also accepts street == 5 with a 5-card board.  Host only. */
int mtt_tree_build_board(const mtt_tree_spec* spec, const uint8_t* board, int32_t nboard,
                         mtt_node* nodes, int32_t capacity, int32_t* n_nodes, int32_t rows[2],
                         int32_t* max_depth);

/* Check a caller-supplied tree (reference FlatNode layout, rows per player as
 * above): offsets in range, children after parents, actions >= 1, no cycles.
 * Host only. */
int mtt_tree_validate(const mtt_node* nodes, int32_t n_nodes, int32_t rows[2]);

/* ------------------------------------------------------------- evaluator */
/* 7 cards per hand (uint8 x 7, packed) -> uint32 score identical to the
 * reference's fast_7card_score (src/tools/mtt_ev_dumper.cu:53-83; copies at
 * honest_multistreet_solver.cu:24-54 and preflop_grid_generator.cu:47-77). */
int mtt_eval7(const uint8_t* d_cards7, uint32_t* d_out, int64_t n, void* stream);

/* Evaluate all C(52,7) hands: d_hist9[k] = hands of category k (score>>24),
 * *d_checksum = sum over hands in colex order of score*(index+1) mod 2^64.
 * If d_key_table (65,536 uint32) is given it receives key -> score for the
 * 16-bit monotone key the scans use; *d_err gets bit 1 if two scores share a
 * key.  No reference kernel: it checks the scorer over every 7-card hand. */
int mtt_eval7_enumerate(uint64_t* d_hist9, uint64_t* d_checksum, uint32_t* d_key_table,
                        int32_t* d_err, void* stream);

/* ------------------------------------------------------ showdown counts */
/* Exact win/tie/loss counts of hero i vs villain j (out[i*H+j], int32) over
 * every completion of a 3-, 4- or 5-card board.  Pairs that share a card or
 * touch the board get zeros.  Replaces kernel_gen_49_turn_matrices
 * (src/postflop/honest_multistreet_solver.cu:56-86), whose float entry is
 * (W + 0.5*T) / (W + T + L) of these counts; its output is villain-major,
 * this one hero-major. */
int mtt_board_showdown_counts(const uint8_t* d_board, int32_t nboard, const uint8_t* d_hands,
                              int32_t H, int32_t* d_w, int32_t* d_t, int32_t* d_l, void* stream);

/* Same counts as mtt_board_showdown_counts, with no device allocation.  No
 * counterpart in the reference.  For callers that may not allocate during the
 * call: a process whose free device memory is already handed to another
 * pool, or a worker loop that must not stall on, or fail in, the allocator.
 * The key scratch is a fixed 1 MiB static device array, one per device.
 * Limit: ceil(C/2) * roundup(H, 64) <= MTT_COUNTS_NOALLOC_MAX_WORDS, where C
 * is the number of board completions (1 river, 48 turn, 1,176 flop), i.e.
 * any H <= 1,326 on 4- and 5-card boards and H <= 384 on 3-card boards;
 * larger sizes return MTT_ERR_UNSUPPORTED before any device work.  The first
 * call on a device looks up the scratch address with that device current;
 * make that first call before any stream capture.  The address is kept per
 * device and context: after a cudaDeviceReset the next call on that device
 * looks it up again in the new context.  Calls that overlap in
 * time on the same device share the scratch and race: order them on one
 * stream or serialise them. */
#define MTT_COUNTS_NOALLOC_MAX_WORDS 262144
int mtt_board_showdown_counts_noalloc(const uint8_t* d_board, int32_t nboard, const uint8_t* d_hands,
                                      int32_t H, int32_t* d_w, int32_t* d_t, int32_t* d_l, void* stream);

/* ------------------------------------------------------------ dumper path */
/* The 1,755 canonical flops with orbit weights, h_out[4*i..] = c1,c2,c3,w
 * (generate_all_1755_flops, src/tools/mtt_ev_dumper.cu:34-51). Host only. */
int mtt_canonical_flops(uint8_t* h_out, int32_t capacity, int32_t* n_out);

/* kernel_evaluate_flop_ev (src/tools/mtt_ev_dumper.cu:85-116) for nflops flops
 * (d_flops: 3 cards each).  d_reach0/1: 1,176 weights over the flop's alive
 * combos in lexicographic order (NULL = uniform 1/1176).  d_ev0/1: [nflops][1176].
 * Bit-exact with the reference. */
int mtt_flop_ev(const uint8_t* d_flops, int32_t nflops, const float* d_reach0,
                const float* d_reach1, float* d_ev0, float* d_ev1, void* stream);

/* ev_dumper's output for nflops flops: d_out [nflops][4][2][169] f32, the
 * per-flop slices of mtt_ev_dump_1755.bin (mtt_ev_dumper.cu:141-173).
 * Bit-exact with the reference's shipped file. */
int mtt_ev_dump(const uint8_t* d_flops, int32_t nflops, float* d_out, void* stream);

/* --------------------------------------------------- heads-up CFR solving */
#define MTT_ALGO_CFRPLUS 0     /* R <- max(0, R + r); S += t * reach * sigma */
#define MTT_ALGO_DCFR    1     /* discount R (alpha/beta) and S (gamma), then add */
#define MTT_SEM_CORRECT   0    /* card removal at showdown and fold, ties split, chance / (N-4) */
#define MTT_SEM_REFERENCE 1    /* the reference kernels' semantics: P1 showdown equity inverted,
                                  no card removal between the hands, chance / (N-2)
                                  (honest_multistreet_solver.cu:163-164,182-187,217) */

typedef struct mtt_solve_params {
    int32_t iters;
    int32_t algo;
    float   alpha, beta, gamma;   /* DCFR only */
    int32_t semantics;
    int32_t threads;              /* CTA size of the sweep kernels (64/128/256); 0 = autotuned.
                                     Results do not depend on it. */
    int32_t exploitability;       /* 1: FP64 best-response pass after the iterations */
    int32_t alternate;            /* 1: alternating updates (CFR+ as published: P0's pass, then
                                     P1's against P0's new strategy); 0: simultaneous updates of
                                     both players per sweep, as the reference kernels do */
    float   avg_power;            /* CFR+ strategy-sum weight t^avg_power (1: linear averaging,
                                     2: quadratic); DCFR uses gamma instead */
    float   target_expl;          /* > 0 (with exploitability = 1 and max_iters > iters): after
                                     `iters` iterations, subgames whose exploitability is above
                                     target_expl (fraction of the starting pot) keep iterating in
                                     chunks of chunk_iters until they pass or reach max_iters */
    int32_t max_iters;
    int32_t chunk_iters;          /* 0: iters / 2 */
} mtt_solve_params;

/* One heads-up subgame.  combos[p] ascending combo ids (0..1325) of player
 * p's range support, none touching the board; ranges[p] their weights. */
typedef struct mtt_subgame {
    const mtt_node* nodes;
    int32_t n_nodes;
    int32_t rows[2];
    uint8_t board[5];
    int32_t nboard;               /* 5 river, 4 turn (river chance nodes), 3 flop (turn then river chance nodes) */
    int32_t H[2];
    const uint16_t* combos[2];
    const float* ranges[2];
} mtt_subgame;

typedef struct mtt_batch mtt_batch;
typedef struct mtt_leafnet mtt_leafnet;   /* the leaf network (declared with its functions below) */

/* Pack n subgames (host pointers) into device memory on the current device.
 * Synchronous.  Per subgame the layout is reach/CFV vectors per node, R and S
 * per regret row, and per-board showdown rank tables. */
int mtt_batch_create(const mtt_subgame* subs, int32_t n, mtt_batch** out);
/* Solve every subgame from zero regrets.  Each iteration is a sequence of
 * level-synchronous launches over the whole batch (forward levels,
 * terminals, backward levels per pass); then, optionally, the FP64
 * best-response pass.  Asynchronous on stream. */
int mtt_batch_solve(mtt_batch* b, const mtt_solve_params* prm, void* stream);
/* Same work as mtt_batch_solve, with one iteration captured as a CUDA graph
 * (on the first call for these params) and replayed per iteration. */
int mtt_batch_solve_graph(mtt_batch* b, const mtt_solve_params* prm, void* stream);
/* Per subgame: [0] BR value of P0, [1] BR of P1, [2] EV of P0 under the
 * average strategies, [3] EV of P1 (per unit of compatible range mass),
 * [4] compatible range mass Z, [5] exploitability (BR0+BR1)/2 / starting pot.
 * Waits for the stream. */
int mtt_batch_results(mtt_batch* b, double* h_out, void* stream);
/* Iterations run per subgame by the last solve (iters, plus continuation
 * chunks when a target exploitability was set).  h_out: n entries. */
int mtt_batch_iterations(mtt_batch* b, int32_t* h_out);
/* Regrets R_p, strategy sums S_p ([rows_p][H_p]) and last-iteration root
 * CFVs (cfv_p[H_p]) of subgame s; any pointer may be NULL.  Synchronous. */
int mtt_batch_read(mtt_batch* b, int32_t s, float* h_R0, float* h_R1, float* h_S0, float* h_S1,
                   float* h_cfv0, float* h_cfv1);
/* Per-node vectors of subgame s after the last iteration: h_reach[n][p][H_p]
 * (player p's reach at node n, from the slot that holds it) and
 * h_cfv[n][p][H_p] (counterfactual values), both [n_nodes][H0 + H1] with
 * player 0's hands first.  Either pointer may be NULL.  Synchronous. */
int mtt_batch_read_vectors(mtt_batch* b, int32_t s, float* h_reach, float* h_cfv);
/* Root values of subgame s from the last FP64 best-response pass (a solve
 * with exploitability = 1): h_ev_p[H_p] = counterfactual values of player
 * p's hands under both average strategies, h_br_p[H_p] = best-response
 * values against the opponent's average strategy.  Any pointer may be NULL.
 * Synchronous. */
int mtt_batch_root_values(mtt_batch* b, int32_t s, double* h_ev0, double* h_ev1, double* h_br0, double* h_br1);
/* Device bytes held, and algorithmic bytes of one CFR iteration over the whole
 * batch (R,S read+write per action-hand; reach and CFV written and read once
 * per player-hand per node). */
int mtt_batch_info(mtt_batch* b, int64_t* device_bytes, int64_t* iter_bytes);
/* Device layout of the per-subgame arrays, for callers that pass their own
 * strategy inputs: h_rows_off[2*s+p] = float offset of player p's rows block
 * of subgame s ([rows_p][Hp_p], Hp_p = H_p rounded up to a multiple of 4,
 * hand i at column i in combos[p] order); h_range_off[s] = float offset of
 * its packed root ranges [Hp_0 | Hp_1]; totals are the array lengths.  Any
 * output may be NULL. */
int mtt_batch_layout(mtt_batch* b, int64_t* h_rows_off, int64_t* h_range_off, int64_t* total_rows,
                     int64_t* total_range);
/* Differentiable EV of fixed strategies, no CFR (no reference counterpart;
 * the values are those of kernel_evaluate_terminals and
 * kernel_backward_sweep, honest_multistreet_solver.cu:128-249, with card
 * removal).  Both players play sigma = softmax(logits) over the actions of
 * every decision node, per hand.  d_logits: [total_rows] in the rows layout;
 * d_ranges: [total_range] packed root ranges (padding 0).  Outputs:
 *   d_ev[s]          = EV of player 0 in chips, sum over compatible hand
 *                      pairs of range0 * range1 * payoff0;
 *   d_grad_ranges    = dEV0/drange in the range layout: [cfv0 | -cfv1] at the
 *                      root (the counterfactual values);
 *   d_grad_logits    = dEV0/dlogits in the rows layout.
 * All device pointers 16-byte aligned.  Overwrites the batch's per-node
 * reach and value vectors (a later solve starts from scratch anyway).
 * Asynchronous; mtt_batch_check reports a bounded-wait failure. */
int mtt_batch_ev_grad(mtt_batch* b, const float* d_logits, const float* d_ranges, float* d_ev,
                      float* d_grad_ranges, float* d_grad_logits, void* stream);
/* Waits for the stream; MTT_ERR_TIMEOUT if a bounded device wait of this
 * batch's kernels gave up since the last solve or ev_grad started. */
int mtt_batch_check(mtt_batch* b, void* stream);
/* Kernels launched for this batch since it was created; a graph replay counts
 * every kernel node it runs. No reference counterpart (instrumentation). */
int mtt_batch_launch_count(mtt_batch* b, int64_t* launches);
/* Batches allocate device memory from a library-owned stream-ordered pool
 * per device that keeps what destroyed batches free, so the next batch of a
 * similar size allocates without mapping new pages.  mtt_trim_pool waits for
 * the current device and returns the kept memory to the driver. */
int mtt_trim_pool(void);
/* Depth-limit leaves (MTT_NODE_LEAF, turn subgames): every pass of every
 * iteration values them by the leaf network `net` (whose batch capacity must
 * hold 48 rows per leaf of the batch) on both players' current reach, per
 * river card, and averages the river cards as a river chance node does
 * (divisor 44, or 46 in the reference semantics).  flags:
 * MTT_LEAF_VALUES_RESIDUAL adds the check-down values of the same ranges to
 * the network's output (a network trained on the residual); net == NULL
 * values the leaves by check-down alone.  Required before solving a batch
 * with leaves; such a batch has no best response (exploitability must be 0),
 * no kernel profile and no ev_grad.  The network stays owned by the caller
 * and must outlive the solves.  No reference counterpart. */
#define MTT_LEAF_VALUES_RESIDUAL 1
int mtt_batch_set_leafnet(mtt_batch* b, mtt_leafnet* net, int32_t flags);
/* Runs `iters` CFR iterations (no best response, no graph) with a CUDA event
 * around each kernel class of every pass and returns, per iteration,
 * h_ms[3] = device time and h_bytes[3] = compulsory bytes (every element a
 * work item reads or writes, counted once) of {forward sweeps, terminal
 * launches, backward sweeps}.  Restarts the batch's solve state.  Blocks.
 * No reference counterpart (instrumentation). */
int mtt_batch_kernel_profile(mtt_batch* b, const mtt_solve_params* prm, int32_t iters, double* h_ms,
                             double* h_bytes, void* stream);
/* Pick the schedule by timing a few iterations of every candidate on this
 * batch: the sweep CTA size (64, 128, 256 threads), the hands per sweep warp
 * item (128 or 256) and the terminals per terminal CTA at most (8 or 16);
 * *threads receives the CTA size (also used when params.threads == 0), the
 * rest stays set on the batch (mtt_batch_schedule).  Results do not depend on
 * the schedule. */
int mtt_batch_autotune(mtt_batch* b, const mtt_solve_params* prm, void* stream, int32_t* threads);
/* Set the schedule: threads 0 (256 unless tuned) or 64/128/256,
 * hands_per_warp 128 or 256, term_chunk 1..16.  Rebuilds the work lists. */
int mtt_batch_set_schedule(mtt_batch* b, int32_t threads, int32_t hands_per_warp, int32_t term_chunk);
int mtt_batch_schedule(mtt_batch* b, int32_t* threads, int32_t* hands_per_warp, int32_t* term_chunk);
/* Waits for the batch's work on the streams it was used with (an event per
 * stream, recorded by each call that launched work), not for the whole
 * device, then returns its memory to the pool in legacy-stream order; another
 * host thread may keep creating or solving other batches meanwhile. */
int mtt_batch_destroy(mtt_batch* b);

/* ------------------------------------------------------ leaf-net GEMM */
#define MTT_GEMM_RELU     1    /* max(0, .) after the bias */
#define MTT_GEMM_OUT_BF16 2    /* C is bf16 (else float) */
#define MTT_GEMM_MASK     4    /* zero C where d_mask (bf16 [M][ldm]) is <= 0: the ReLU backward */
/* C[M x N] = A[M x K] * B[N x K]^T (+ d_bias[N]) on the tcgen05 tensor cores,
 * BF16 inputs, FP32 accumulation.  A, B row-major with row strides lda, ldb
 * (elements, multiples of 8; base addresses 16-byte aligned); C row stride
 * ldc.  d_err: device int, bit 0 set if a bounded wait gave up.  No
 * reference counterpart (the reference has no learned component). */
int mtt_gemm_bf16(const void* d_A, int32_t lda, const void* d_B, int32_t ldb, void* d_C, int32_t ldc,
                  int32_t M, int32_t N, int32_t K, const float* d_bias, const void* d_mask, int32_t ldm,
                  int32_t flags, int32_t* d_err, void* stream);
/* The same with a caller-owned FP32 workspace of ws_floats floats on the
 * stream's device.  A product of fewer output tiles (128 x 256) than about
 * the SM count over at least 512 of K is split along K so that the splits
 * fill the SMs: each split writes its partial tile to d_ws, and a second
 * kernel adds the splits in a fixed order and applies the epilogue.  The
 * split count is lowered until splits x M x N fits ws_floats; with none left
 * (or d_ws null) it is mtt_gemm_bf16.  Results are deterministic; they
 * differ from the one-pass kernel's in FP32 summation order only.  d_ws must
 * not be used by anything else until the call's work on the stream is done. */
int mtt_gemm_bf16_ws(const void* d_A, int32_t lda, const void* d_B, int32_t ldb, void* d_C, int32_t ldc,
                     int32_t M, int32_t N, int32_t K, const float* d_bias, const void* d_mask, int32_t ldm,
                     int32_t flags, int32_t* d_err, float* d_ws, int64_t ws_floats, void* stream);

/* ------------------------------------------------------ leaf network */
/* MLP for depth-limited solving (no reference counterpart): features
 * [ranges of both players over the 1,326 combos | board one-hot (52) | pot |
 * stack] = 2,706 -> 3 x 1,024 ReLU -> 2,652 counterfactual values (both
 * players' 1,326 combos, in units of the pot).  BF16 weights and
 * activations, FP32 accumulation and FP32 master weights (Adam). */
#define MTT_LEAF_IN     2706
#define MTT_LEAF_HIDDEN 1024
#define MTT_LEAF_OUT    2652
#define MTT_LEAF_ZERO_OUTPUT 1   /* flags: start the output layer at zero (a residual on a base estimate) */
/* batch_cap: largest batch (multiple of 8).  He-initialised from seed. */
int mtt_leafnet_create(int32_t batch_cap, uint64_t seed, int32_t flags, mtt_leafnet** out);
/* d_x [M][2706] float features -> d_y [M][2652] float predictions. */
int mtt_leafnet_forward(mtt_leafnet* n, const float* d_x, int32_t M, float* d_y, void* stream);
/* *cap = the largest batch (rows) the network was created for. */
int mtt_leafnet_capacity(mtt_leafnet* n, int32_t* cap);
/* Gradients of the masked mean squared error sum(w (y - t)^2) / (M * 2652)
 * for targets d_t [M][2652] and weights d_w (NULL = all ones); *h_loss gets
 * the loss (synchronises when h_loss is given).  M a multiple of 8. */
int mtt_leafnet_gradients(mtt_leafnet* n, const float* d_x, const float* d_t, const float* d_w, int32_t M,
                          double* h_loss, void* stream);
/* Gradients as above, then one Adam step (beta1 0.9, beta2 0.999, eps 1e-8). */
int mtt_leafnet_train_step(mtt_leafnet* n, const float* d_x, const float* d_t, const float* d_w, int32_t M,
                           float lr, double* h_loss, void* stream);
/* Layer l (0..3) parameters and last gradients in the padded shape
 * shape[0] x shape[1] = out x in (input 2,752 and output 2,688 columns,
 * padding zero).  Any pointer may be NULL.  Synchronous. */
int mtt_leafnet_params(mtt_leafnet* n, int32_t layer, float* h_w, float* h_b, float* h_gw, float* h_gb,
                       int32_t* shape);
/* MTT_ERR_TIMEOUT if a bounded wait in the network's GEMMs gave up. */
int mtt_leafnet_check(mtt_leafnet* n);
int mtt_leafnet_destroy(mtt_leafnet* n);
/* Check-down leaf values, the estimate the leaf network corrects: for n river
 * boards (d_boards [n][5]) and both players' ranges over the 1,326 combos
 * (d_range0, d_range1 [n][1326], each summing to 1 over the combos that avoid
 * the board), d_out[b][p][h] = the value of player p's combo h in units of
 * the pot when both check the river down: half of the opponent's compatible
 * mass below it minus half of the mass above it (card removal, split ties).
 * Combos touching the board get 0.  No reference counterpart. */
int mtt_checkdown_values(const uint8_t* d_boards, const float* d_range0, const float* d_range1, int32_t n,
                         float* d_out, void* stream);

/* ------------------------------------------------- preflop anchor chain */
#define MTT_PF_REFERENCE 0   /* the reference's arithmetic, quirks included (see preflop.cu) */
#define MTT_PF_CORRECT   1   /* valid class cards, sampling without replacement, every
                                flop-compatible combo, ties count one half */
/* 169 x 169 all-in equities of the hand classes, d_out[h*169 + v]
 * (kernel_gen_preflop_matrix, src/preflop/preflop_grid_generator.cu:95-127:
 * 3,000 LCG board samples per pair); d_wins / d_ties (optional, together)
 * receive the integer counts. */
int mtt_pf_allin_matrix(int32_t mode, float* d_out, int32_t* d_wins, int32_t* d_ties, void* stream);
/* Class-reduced flop equity matrices of n flops (3 cards each):
 * d_out[f][v][h] (kernel_gen_100_flop_matrices + kernel_reduce_combo_to_class_matrices,
 * preflop_grid_generator.cu:130-223), without the 1,216 x 1,216 combo
 * matrices of every flop resident at once. */
int mtt_pf_flop_class_matrices(int32_t mode, const uint8_t* d_flops, int32_t n, float* d_out, void* stream);
typedef struct mtt_pf_params {
    int32_t iters;       /* 500 in the reference */
    float   stack_bb;    /* 20 */
    float   bubble;      /* 1.35 */
    float   dead_pot;    /* 2.5 */
} mtt_pf_params;
/* DCFR over the closed BTN-vs-BB preflop tree (kernel_cosolve_100_board_matrices,
 * kernel_build_closed_preflop_cfvs, kernel_dcfr_step, kernel_update_dynamic_reaches
 * and the loop at preflop_grid_generator.cu:228-421,588-614).  d_sums / d_sigma
 * ([10][192]): strategy sums / last strategies of the nodes BTN root (fold,
 * min-raise, jam), BB vs min-raise (fold, call, 3-bet jam), BTN vs 3-bet (fold,
 * call), BB vs open jam (fold, call), one 192-wide row per action. */
int mtt_pf_dcfr(const float* d_flop_weights, const float* d_class_mats, int32_t n_flops, const float* d_allin,
                const mtt_pf_params* p, float* d_sums, float* d_sigma, void* stream);
/* Read a flop-subset file (uint32 count, then per flop c1, c2, c3, pad, float
 * weight; preflop_grid_generator.cu:446-459).  path NULL: data/mtt_subset.bin,
 * then ./mtt_subset.bin.  h_flops NULL: only *n.  Host only. */
int mtt_pf_read_subset(const char* path, uint8_t* h_flops, float* h_weights, int32_t capacity, int32_t* n);
/* Class (0..168) of the combo c1 < c2 as the reference numbers them (pairs AA..22,
 * suited, offsuit); -1 if invalid. */
int mtt_pf_combo_class(int32_t c1, int32_t c2);

/* ------------------------------------------- flop subset (NN-OMP, FP64) */
/* Greedy non-negative orthogonal matching pursuit over the columns of a
 * flop-major matrix, replacing scripts/optimize_subset.py:29-50 (which
 * produces data/mtt_subset.bin from mtt_ev_dump_1755.bin).  Column j is
 * d_cols[j * nfeat .. + nfeat) (the dump read as [1755][1352] f32 is the
 * reference's A^T); d_colw: ncols FP64 column weights (the orbit weights of
 * mtt_canonical_flops).  The target is b = A colw / sum(colw).  Each of the
 * nselect steps adds the unselected column with the largest <A_j, r> / |A_j|
 * (the first on ties), then refits the non-negative least-squares weights of
 * all selected columns to b (Lawson-Hanson, FP64) and sets r = b - A_sel x.
 * Writes d_idx[nselect] (selection order) and d_w[nselect], the last fit's
 * weights scaled to sum to ncols.  Same selections as the reference on the
 * shipped dump, and weights within FP64 rounding of scipy's.  Inputs must be
 * finite.  nselect <= min(ncols, MTT_SUBSET_MAX_SELECT).  Returns
 * MTT_ERR_UNSUPPORTED if a least-squares subproblem is rank-deficient or takes
 * more than 3 * (columns) passive-set solves (scipy.optimize.nnls raises for
 * the latter).  Synchronises the stream. */
#define MTT_SUBSET_MAX_SELECT 128
int mtt_subset_nnomp(const float* d_cols, int32_t ncols, int32_t nfeat, const double* d_colw,
                     int32_t nselect, int32_t* d_idx, double* d_w, void* stream);
/* Write a selection as the reference does (optimize_subset.py:52-65): bin_path
 * gets uint32 n, then per flop c1, c2, c3, 0 (u8) and the weight as f32;
 * txt_path gets one "<card><card><card>:<weight %.4f>" line per flop (cards
 * as "As", "Td", ...).  h_flops3: 3 cards per flop.  Either path may be NULL.
 * Host only. */
int mtt_subset_write(const char* bin_path, const char* txt_path, const uint8_t* h_flops3, const double* h_w,
                     int32_t n);

/* ------------------------------------------- ICM (Malmuth-Harville, FP64) */
/* Tournament equity of n seats with chip stacks[n] and m payouts[m] (prize
 * for 1st, 2nd, ...): the probability that seat i finishes k-th is the
 * Malmuth-Harville product of stack shares; out[i] = sum_k payouts[k] *
 * P(i finishes k-th).  n <= 16, m <= n.  Host only.  No reference
 * counterpart: the reference takes bubble factors as input
 * (multiway_4way_engine.cu:85, bubble_factors[4x4]). */
int mtt_icm_equity(const double* stacks, int32_t n, const double* payouts, int32_t m, double* out);
/* Bubble factors of the players in a hand: seats[k] (k < np <= 4) index the
 * n seats.  For k != j: risk X = min(stack of k, stack of j);
 *   bf[k*np + j] = (E_k(now) - E_k(k loses X to j)) / (E_k(k wins X from j) - E_k(now)),
 * and bf[k*np + k] = the mean of bf[k*np + j] over j != k (k against the
 * field).  These are the bubble_factors the multiway terminals scale losses
 * by.  Host only. */
int mtt_icm_bubble_factors(const double* stacks, int32_t n, const double* payouts, int32_t m,
                           const int32_t* seats, int32_t np, double* bf);

/* ---------------------------------------------------- multiway (4 players) */
#define MTT_MW_PLAYERS 4
#define MTT_MW_MAX_ACTIONS 3   /* as the reference engine (MAX_POST_ACTIONS, multiway_4way_engine.cu:14) */
/* Flat 4-player node, 32 bytes, the reference's 4-way FlatNode
 * (multiway_4way_engine.cu:20-24): fold terminals keep the single remaining
 * player's bit in active_mask; showdown terminals the bits of the players
 * still in.  As in the heads-up layout, infoset_offset is the first row of
 * this node in its player's own regret array. */
typedef struct mtt_mw_node {
    uint8_t  type;
    uint8_t  player;
    uint8_t  num_actions;
    uint8_t  active_mask;
    int32_t  children_offset;
    int32_t  infoset_offset;
    float    pot_size;
    float    committed[4];
} mtt_mw_node;

/* Single-street 4-player betting: players act in seat order 0..3; with no
 * bet a player checks or bets one of bet_sizes (fractions of the pot); facing
 * a bet a player folds, calls or (while fewer than raise_cap raises were
 * made) raises raise_size * (pot + to_call) on top of the call.  Bets are
 * capped at the player's remaining stack.  The round closes when every
 * player still in has acted and matched the bet.  At most 3 actions per
 * node. */
typedef struct mtt_mw_spec {
    float   pot;                  /* dead money already in (split equally into committed[]) */
    float   stacks[4];            /* chips behind per player */
    int32_t n_bet_sizes;          /* 1 or 2 */
    float   bet_sizes[2];
    float   raise_size;
    int32_t raise_cap;
} mtt_mw_spec;

int mtt_mw_tree_build(const mtt_mw_spec* spec, mtt_mw_node* nodes, int32_t capacity, int32_t* n_nodes,
                      int32_t rows[4], int32_t* max_depth);

/* One 4-player river subgame: every player's range is over the same H
 * ascending combo ids (the reference's shared combo axis), none touching the
 * board; bubble[16] = loss multipliers bf[p*4 + w] (row p loses to w; the
 * diagonal is p against the field), 1 = chip EV. */
typedef struct mtt_mw_subgame {
    const mtt_mw_node* nodes;
    int32_t n_nodes;
    int32_t rows[4];
    uint8_t board[5];
    int32_t H;
    const uint16_t* combos;
    const float* ranges[4];
    float bubble[16];
} mtt_mw_subgame;

typedef struct mtt_mw_batch mtt_mw_batch;

int mtt_mw_batch_create(const mtt_mw_subgame* subs, int32_t n, mtt_mw_batch** out);
/* CFR+ (or DCFR) with simultaneous updates of all four players, as the
 * reference kernels (kernel_4way_forward_sweep / _evaluate_terminals /
 * _backward_cfr_plus, multiway_4way_engine.cu:41-257).  Uses iters, algo,
 * alpha/beta/gamma, semantics (MTT_SEM_REFERENCE: the reference's strict
 * rank-position order, no ties, no card removal; MTT_SEM_CORRECT: each
 * player's hand removes its two cards from every opponent's range and equal
 * hands split the pot; opponents are not conditioned on one another), avg_power;
 * one iteration is captured as a CUDA graph when graph != 0.  Asynchronous. */
int mtt_mw_batch_solve(mtt_mw_batch* b, const mtt_solve_params* prm, int32_t graph, void* stream);
/* Per subgame and player, the EV of that player's range (chips) under the
 * average strategies: h_out[s*4 + p].  Synchronous. */
int mtt_mw_batch_values(mtt_mw_batch* b, double* h_out, void* stream);
/* R_p, S_p ([rows_p][H]) and the last iteration's root CFVs ([4][H]) of
 * subgame s; any pointer may be NULL.  Synchronous. */
int mtt_mw_batch_read(mtt_mw_batch* b, int32_t s, float* h_R[4], float* h_S[4], float* h_cfv);
int mtt_mw_batch_destroy(mtt_mw_batch* b);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* MTT_B200_H */
