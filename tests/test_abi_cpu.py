"""C ABI and host logic that run without a GPU: exports, trees, validation."""
import ctypes
import re

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(mtt):
    import subprocess
    L = mtt.lib()
    declared = mtt._lib.exported_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", mtt._lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mtt_\w+)", out))
    assert set(declared) <= exported
    assert mtt.lib().mtt_version().startswith(b"mtt-b200")
    assert mtt.lib().mtt_status_string(0) == b"ok"


def _check_tree(mtt, nodes, rows):
    assert mtt.validate_tree(nodes, rows) == 0
    n = len(nodes)
    seen = np.zeros(n, bool)
    for i, nd in enumerate(nodes):
        if nd["type"] in (mtt.NODE_DECISION, mtt.NODE_CHANCE):
            f, a = nd["children_offset"], nd["num_actions"]
            assert f > i and f + a <= n
            assert not seen[f:f + a].any()
            seen[f:f + a] = True
            for c in range(f, f + a):
                assert nodes[c]["depth"] == nd["depth"] + 1
        if nd["type"] == mtt.NODE_SHOWDOWN:
            assert abs(nd["committed"][0] - nd["committed"][1]) < 1e-3
        if nd["type"] != mtt.NODE_CHANCE:
            assert abs(nd["pot_size"] - nd["committed"].sum()) < 1e-3
    assert seen[1:].all()


def test_river_tree_config0_shape(mtt):
    nodes, rows, depth = mtt.build_tree(100, 200, [0.5, 1.0], raise_cap=1)
    _check_tree(mtt, nodes, rows)
    assert nodes[0]["num_actions"] == 4            # check, 50, 100, all-in
    assert nodes[0]["player"] == 0
    assert rows[0] == rows[1]
    # fold payoffs are zero-sum: winner gains the loser's commitment
    for nd in nodes[nodes["type"] == mtt.NODE_FOLD]:
        w = 0 if nd["active_mask"] == 1 else 1
        assert nd["pot_size"] - nd["committed"][w] == pytest.approx(nd["committed"][1 - w])
    # all-in never exceeds the stack
    assert (nodes["committed"] <= 50 + 200 + 1e-3).all()


@pytest.mark.parametrize("sizes,cap,pot,stack", [([0.853], 1, 37.8, 31.8), ([0.25, 0.5, 1.0, 2.0], 3, 20, 240),
                                                 ([1.992], 3, 144.5, 1195.0), ([0.347, 0.579, 1.525], 2, 138.3, 964)])
def test_river_tree_random_specs(mtt, sizes, cap, pot, stack):
    nodes, rows, depth = mtt.build_tree(pot, stack, sizes, raise_cap=cap)
    _check_tree(mtt, nodes, rows)
    assert nodes["num_actions"].max() <= 8


def test_turn_tree_has_river_chance_layer(mtt):
    board = [0, 13, 26, 39]
    nodes, rows, depth = mtt.build_tree(60, 470, [0.33, 0.75, 1.5], raise_cap=2, street=4, board=board)
    _check_tree(mtt, nodes, rows)
    ch = nodes[nodes["type"] == mtt.NODE_CHANCE]
    assert len(ch) > 0 and (ch["num_actions"] == 48).all()
    for nd in ch:
        kids = nodes[nd["children_offset"]:nd["children_offset"] + 48]
        assert sorted(kids["turn_idx"].tolist()) == [c for c in range(52) if c not in board]


def test_validation_rejects_malformed_trees(mtt):
    nodes, rows, _ = mtt.build_tree(100, 200, [0.5, 1.0], raise_cap=1)
    bad = nodes.copy(); bad[0]["children_offset"] = 0
    assert mtt.validate_tree(bad, rows) != 0                   # child before parent / cycle
    bad = nodes.copy(); bad[0]["children_offset"] = len(nodes) - 1
    assert mtt.validate_tree(bad, rows) != 0                   # children out of range
    bad = nodes.copy(); bad[0]["infoset_offset"] = rows[0]
    assert mtt.validate_tree(bad, rows) != 0                   # regret rows out of range
    bad = nodes.copy(); bad[nodes["type"] == mtt.NODE_FOLD][0]["active_mask"] = 3
    i = int(np.nonzero(nodes["type"] == mtt.NODE_FOLD)[0][0]); bad = nodes.copy(); bad[i]["active_mask"] = 3
    assert mtt.validate_tree(bad, rows) != 0
    assert mtt.validate_tree(nodes, rows) == 0


def test_invalid_arguments_return_status_not_crash(mtt):
    L = mtt.lib()
    assert L.mtt_eval7(None, None, -1, None) == 1
    assert L.mtt_board_showdown_counts(None, 7, None, 10, None, None, None, None) == 1
    assert L.mtt_batch_create(None, 0, None) == 1
    assert L.mtt_batch_solve(None, None, None) == 1
    sp = mtt.make_spec(-1, 100, [0.5])
    n = ctypes.c_int32(); rows = (ctypes.c_int32 * 2)(); d = ctypes.c_int32()
    assert L.mtt_tree_build(ctypes.byref(sp), None, 0, ctypes.byref(n), rows, ctypes.byref(d)) == 1


def test_canonical_flops_host(mtt, orc):
    assert (mtt.canonical_flops() == orc.gen_flops()).all()


def test_workload_config2_shapes(wl):
    subs = wl.river_batch(n=64, seed=2)
    assert len(subs) == 64
    for g in subs:
        for p in (0, 1):
            c = g[f"combos{p}"]
            assert 200 <= len(c) <= 1081 and (np.diff(c.astype(int)) > 0).all()
            assert (g[f"range{p}"] > 0).all()
        assert g["nodes"]["num_actions"].max() <= 8


def test_turn_tree_with_river_leaves(mtt):
    """Turn rounds that close with chips behind end in NODE_LEAF (chips
    behind in `reserved`); all-in closes still deal the river to showdowns."""
    board = [14, 26, 41, 31]
    full, rows_f, _ = mtt.build_tree(100.0, 150.0, [0.5, 1.0], raise_cap=1, street=4, board=board)
    lim, rows_l, _ = mtt.build_tree(100.0, 150.0, [0.5, 1.0], raise_cap=1, street=4, board=board, river_leaves=True)
    assert mtt.validate_tree(lim, rows_l) == 0
    leaves = lim[lim["type"] == mtt.NODE_LEAF]
    assert len(leaves) == 5
    assert sorted({round(float(r) / float(p), 6) for r, p in zip(leaves["reserved"], leaves["pot_size"])}) == \
        [0.166667, 0.5, 1.5]
    assert np.all(leaves["committed"][:, 0] == leaves["committed"][:, 1])
    # the leaf tree keeps the turn rows and drops the river ones
    n_dec_turn = int(np.sum((lim["type"] == mtt.NODE_DECISION)))
    assert rows_l[0] + rows_l[1] < rows_f[0] + rows_f[1] and n_dec_turn == 12
    # every leaf of the limited tree is a river chance node of the full tree
    assert int(np.sum(full["type"] == mtt.NODE_CHANCE)) == len(leaves) + int(np.sum(lim["type"] == mtt.NODE_CHANCE))
    with pytest.raises(mtt.MttError):
        mtt.build_tree(100.0, 150.0, [0.5], street=5, river_leaves=True)


def test_flop_tree_turn_chance_and_river_runout(mtt):
    """Flop trees: flop betting, a 49-card turn chance layer, turn betting,
    then a 48-card river chance layer straight to showdowns; every showdown
    sits below both deals."""
    board = [3, 17, 42]
    nodes, rows, depth = mtt.build_tree(100.0, 150.0, [0.5, 1.0], raise_cap=1, street=3, board=board)
    assert mtt.validate_tree(nodes, rows) == 0
    n = len(nodes)
    parent = np.full(n, -1)
    for i, nd in enumerate(nodes):
        if nd["type"] in (mtt.NODE_DECISION, mtt.NODE_CHANCE):
            parent[nd["children_offset"]:nd["children_offset"] + nd["num_actions"]] = i
    deals = np.zeros(n, int)
    for i in range(1, n):
        deals[i] = deals[parent[i]] + (nodes[parent[i]]["type"] == mtt.NODE_CHANCE)
    chance = nodes["type"] == mtt.NODE_CHANCE
    assert set(nodes["num_actions"][chance & (deals == 0)]) == {49}
    assert set(nodes["num_actions"][chance & (deals == 1)]) == {48}
    assert np.all(deals[nodes["type"] == mtt.NODE_SHOWDOWN] == 2)
    # no river betting: every child of a river chance node is a showdown
    for i in np.nonzero(chance & (deals == 1))[0]:
        c0 = nodes[i]["children_offset"]
        assert np.all(nodes["type"][c0:c0 + nodes[i]["num_actions"]] == mtt.NODE_SHOWDOWN)
    with pytest.raises(mtt.MttError):
        mtt.build_tree(100.0, 150.0, [0.5], street=3, board=[3, 17, 42, 5])


def test_command_line_drivers_build_and_print_usage():
    """The reference's executables (Makefile: ev_dumper, preflop_gen,
    hu_solver, multiway_solver) and its subset script (subset_optimizer),
    built over the C ABI; --help needs no GPU."""
    import importlib.util
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("mtt_build", os.path.join(root, "mtt-gpu-solver_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    exes = b.build_drivers(quiet=True)
    assert sorted(os.path.basename(e) for e in exes) == ["ev_dumper", "hu_solver", "multiway_solver", "preflop_gen",
                                                                  "subset_optimizer"]
    for e in exes:
        r = subprocess.run([e, "--help"], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0 and r.stdout.startswith("usage: " + os.path.basename(e)), (e, r.stdout, r.stderr)
