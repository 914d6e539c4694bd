"""The C ABI's showdown counts pinned to the reference's own kernel.

oracle/_ref/ref_turn_matrices is built by `make -C oracle ref` from the
reference's source file (src/postflop/honest_multistreet_solver.cu) and runs
its kernel_gen_49_turn_matrices (:56-86) for one flop.  Each of its entries is
(wins + 0.5f * ties) / rivers in f32, or 0 for a pair that shares a card or
touches the turn.  The same f32 expression formed from mtt_board_showdown_counts
on each of the 49 turn boards must give the same bits, for every hero and
villain.  Skipped where the checker was not built (no reference sources)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_turn_matrices")
NPAD = 1216


@pytest.mark.parametrize("flop", [(51, 46, 23), (0, 1, 20), (4, 8, 12)])
def test_turn_counts_match_reference_kernel(mtt, cuda, tmp_path, flop):
    import torch
    if not os.path.isfile(REF_BIN):
        pytest.skip("oracle/_ref/ref_turn_matrices not built (needs the reference sources)")
    out = tmp_path / "turn.f32"
    r = subprocess.run([REF_BIN, *map(str, flop), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.memmap(out, dtype="<f4", mode="r", shape=(49, NPAD, NPAD))
    deck = [c for c in range(52) if c not in flop]
    hands = np.array([(a, b) for i, a in enumerate(deck) for b in deck[i + 1:]], dtype=np.uint8)
    H = len(hands)
    assert H == 1176
    hd = torch.from_numpy(hands).to(cuda)
    for t, turn in enumerate(deck):
        board = torch.tensor(list(flop) + [turn], dtype=torch.uint8, device=cuda)
        W, T, L = (x.cpu().numpy() for x in mtt.board_showdown_counts(board, hd))
        tot = W + T + L
        with np.errstate(divide="ignore", invalid="ignore"):
            eq = (W.astype(np.float32) + np.float32(0.5) * T.astype(np.float32)) / tot.astype(np.float32)
        eq = np.where(tot > 0, eq, np.float32(0.0)).astype(np.float32)
        got = np.ascontiguousarray(ref[t, :H, :H]).T          # the reference is villain-major
        assert np.array_equal(got.view(np.uint32), eq.view(np.uint32)), (flop, turn)
        # padding villain slots are written as zeros, hero padding is never written
        assert not np.any(ref[t, H:, :H])


@pytest.mark.parametrize("iters", [1, 4])
def test_solver_matches_reference_sweep_kernels(mtt, cuda, iters):
    # the batched solver in the reference semantics (simultaneous updates,
    # linear averaging) against the reference's own sweep kernels, through the
    # fixture tests/golden/make_ref_hu_golden.py made with them on a B200
    import test_oracle_ref_hu as fx
    sub, want = fx.load_fixture()
    b = mtt.RiverBatch([sub])
    b.solve(mtt.solve_params(iters=iters, algo=0, semantics=1, alternate=False, avg_power=1.0, threads=128,
                             exploitability=False))
    got = b.read(0)
    b.close()
    fx.compare(sub, want[iters], got)


@pytest.mark.parametrize("iters", [1, 4])
def test_multiway_solver_matches_reference_kernels(mtt, cuda, iters):
    # the four-player solver in the reference semantics against the reference's
    # own four-player kernels, through tests/golden/make_ref_mw_golden.py's fixture
    import importlib
    import test_oracle_ref_mw as fx
    mw = importlib.import_module("mtt-gpu-solver_b200.multiway")
    sub, want = fx.load_fixture()
    b = mw.MultiwayBatch([sub])
    b.solve(mtt.solve_params(iters=iters, algo=0, semantics=1, avg_power=1.0))
    got = b.read(0)
    b.close()
    fx.compare(sub, want[iters], got)
