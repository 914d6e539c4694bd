"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: boards, ranges and betting abstractions are
drawn from numpy's PCG64 generator with a fixed seed.

* river_uniform (config 0): one HU river subgame, 5-card board from the seed,
  both ranges uniform over the 1,081 board-compatible combos, pot 100, stack
  200, bets {50%, 100%} + all-in, one raise.
* river_batch (config 2): n uneven river subgames; per subgame 1-4 bet sizes
  from U[25%, 200%], raise cap 1-3, supports of 200-1,081 combos with
  lognormal(0, 1) weights, pot U[20, 200], SPR U[0.5, 12].
* diff_boards (config 3): n seeded river boards with the config-0 tree and
  uniform ranges, plus N(0, 1) strategy logits per node and hand.
"""
import numpy as np

from . import build_tree, live_combos


def draw_board(rng, n=5):
    return [int(c) for c in rng.choice(52, size=n, replace=False)]


def _tree_cached(cache, pot, stack, sizes, cap, street=5, board=None):
    key = (round(float(pot), 6), round(float(stack), 6), tuple(round(float(s), 6) for s in sizes), int(cap), street,
           tuple(board) if board is not None else None)
    t = cache.get(key)
    if t is None:
        t = build_tree(pot, stack, list(sizes), raise_cap=cap, street=street, board=board)
        cache[key] = t
    return t


def river_uniform(seed=0, pot=100.0, stack=200.0, bet_sizes=(0.5, 1.0), raise_cap=1, n_hands=None):
    """Config 0.  n_hands (optional) restricts both ranges to the first
    n_hands live combos (small parity cases)."""
    rng = np.random.default_rng(seed)
    board = draw_board(rng)
    live = live_combos(board)
    if n_hands is not None:
        live = np.sort(rng.choice(live, size=n_hands, replace=False)).astype(np.uint16)
    nodes, rows, _ = build_tree(pot, stack, list(bet_sizes), raise_cap=raise_cap)
    r = np.full(len(live), 1.0 / len(live), dtype=np.float32)
    return {"nodes": nodes, "rows": rows, "board": board, "combos0": live, "combos1": live.copy(),
            "range0": r, "range1": r.copy(), "pot": pot}


def river_batch(n=4096, seed=2, min_support=200, max_support=1081, max_sizes=4):
    """Config 2 (the batched uneven river workload)."""
    rng = np.random.default_rng(seed)
    cache = {}
    subs = []
    for _ in range(n):
        board = draw_board(rng)
        live = live_combos(board)
        nsz = int(rng.integers(1, max_sizes + 1))
        sizes = np.sort(rng.uniform(0.25, 2.0, size=nsz)).round(3)
        cap = int(rng.integers(1, 4))
        pot = float(np.round(rng.uniform(20.0, 200.0), 1))
        spr = float(np.round(rng.uniform(0.5, 12.0), 2))
        stack = float(np.round(pot * spr, 1))
        nodes, rows, _ = _tree_cached(cache, pot, stack, sizes, cap)
        g = {"nodes": nodes, "rows": rows, "board": board, "pot": pot}
        for p in (0, 1):
            k = int(rng.integers(min_support, min(max_support, len(live)) + 1))
            sup = np.sort(rng.choice(live, size=k, replace=False)).astype(np.uint16)
            w = rng.lognormal(0.0, 1.0, size=k).astype(np.float32)
            g[f"combos{p}"] = sup
            g[f"range{p}"] = w
        subs.append(g)
    return subs


def diff_boards(n=1024, seed=3, n_hands=None):
    """Config 3 (differentiable EV): n river subgames with config-0 trees
    (pot 100, stack 200, bets {50%, 100%} + all-in, one raise) on boards drawn
    from the seed, uniform ranges over the board's live combos (or n_hands of
    them), and logits [rows_p][H_p] drawn N(0, 1) per node and hand."""
    rng = np.random.default_rng(seed)
    nodes, rows, _ = build_tree(100.0, 200.0, [0.5, 1.0], raise_cap=1)
    subs, logits = [], []
    for _ in range(n):
        board = draw_board(rng)
        live = live_combos(board)
        if n_hands is not None:
            live = np.sort(rng.choice(live, size=n_hands, replace=False)).astype(np.uint16)
        r = np.full(len(live), 1.0 / len(live), dtype=np.float32)
        subs.append({"nodes": nodes, "rows": rows, "board": board, "combos0": live, "combos1": live.copy(),
                     "range0": r, "range1": r.copy(), "pot": 100.0})
        logits.append((rng.standard_normal((int(rows[0]), len(live))).astype(np.float32),
                       rng.standard_normal((int(rows[1]), len(live))).astype(np.float32)))
    return subs, logits


def multiway_icm(seed=4, n_hands=None, pot_bb=4.0, raise_cap=2):
    """Config 4 (four-player ICM river): eight seats with stacks drawn
    lognormal(log 20 bb, 0.5); seats 0-3 are in the hand; payouts 50/30/20;
    Malmuth-Harville bubble factors (FP64, host); a seeded river board;
    Dirichlet(0.3) ranges over the 1,326 combos with board-blocked combos
    removed (the live combos, or n_hands of them); the tree has bets {50%,
    100%} and one raise size (pot), re-raised up to raise_cap times (1,585
    nodes at seed 4's stacks; 677 with a single raise), pot_bb of dead
    money."""
    from . import multiway as mw
    rng = np.random.default_rng(seed)
    stacks = rng.lognormal(np.log(20.0), 0.5, size=8)
    payouts = [0.5, 0.3, 0.2]
    bf = mw.bubble_factors(stacks, payouts, [0, 1, 2, 3])
    board = draw_board(rng)
    live = live_combos(board)
    if n_hands is not None:
        live = np.sort(rng.choice(live, size=n_hands, replace=False)).astype(np.uint16)
    behind = [float(np.round(s - pot_bb / 4, 3)) for s in stacks[:4]]
    nodes, rows, _ = mw.build_tree(pot_bb, behind, [0.5, 1.0], 1.0, raise_cap)
    ranges = []
    for _ in range(4):
        w = rng.dirichlet(np.full(1326, 0.3))[live.astype(np.int64)]
        ranges.append((w / w.sum()).astype(np.float32))
    return {"nodes": nodes, "rows": rows, "board": board, "combos": live, "ranges": ranges, "bubble": bf,
            "pot": pot_bb, "stacks": stacks, "payouts": payouts}


def turn_dcfr(seed=1, n_hands=None):
    """Config 1 (heads-up turn + river DCFR): a 4-card turn board from the
    seed, 48 river cards; each player's range is a 1,326-entry Dirichlet(0.3)
    weight vector with board-blocked combos removed (or n_hands of the live
    combos); pot 60, stack 470; bets {33%, 75%, 150%} + all-in, 2 raises,
    on both streets."""
    rng = np.random.default_rng(seed)
    board = draw_board(rng, 4)
    live = live_combos(board)
    nodes, rows, _ = build_tree(60.0, 470.0, [0.33, 0.75, 1.5], raise_cap=2, street=4, board=board)
    g = {"nodes": nodes, "rows": rows, "board": board, "pot": 60.0}
    for p in (0, 1):
        w = rng.dirichlet(np.full(1326, 0.3))
        c = live if n_hands is None else np.sort(rng.choice(live, size=n_hands, replace=False)).astype(np.uint16)
        r = w[c.astype(np.int64)]
        g[f"combos{p}"] = c.astype(np.uint16)
        g[f"range{p}"] = (r / r.sum()).astype(np.float32)
    return g


def flop_runout(seed=6, n_hands=None, pot=100.0, stack=150.0, bet_sizes=(0.5, 1.0), raise_cap=1, alpha=0.3):
    """A heads-up flop subgame with the reference's multistreet structure
    (honest_multistreet_solver.cu:97-104,205-219): flop betting, 49 turn
    cards, turn betting, then the river run out to showdowns.  A seeded
    3-card flop; each player's range is a 1,326-entry Dirichlet(alpha)
    weight vector with flop-blocked combos removed (or n_hands of the live
    combos)."""
    rng = np.random.default_rng(seed)
    board = draw_board(rng, 3)
    live = live_combos(board)
    nodes, rows, _ = build_tree(pot, stack, list(bet_sizes), raise_cap=raise_cap, street=3, board=board)
    g = {"nodes": nodes, "rows": rows, "board": board, "pot": float(pot)}
    for p in (0, 1):
        w = rng.dirichlet(np.full(1326, alpha))
        c = live if n_hands is None else np.sort(rng.choice(live, size=n_hands, replace=False)).astype(np.uint16)
        r = w[c.astype(np.int64)]
        g[f"combos{p}"] = c.astype(np.uint16)
        g[f"range{p}"] = (r / r.sum()).astype(np.float32)
    return g
