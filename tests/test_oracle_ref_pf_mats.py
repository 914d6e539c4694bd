"""The preflop class matrices against the reference's own kernels.

tests/golden/ref_pf_flop_mats.npz holds the class-reduced flop matrices that
the reference's kernel_gen_100_flop_matrices and
kernel_reduce_combo_to_class_matrices (src/preflop/preflop_grid_generator.cu:128-223),
built with its own --use_fast_math, produced on a B200 for the first three
flops of the shipped subset (made by tests/golden/make_ref_pf_mats_golden.py).
The oracle's reference mode (bit-exact with the GPU's, full-size hashes in
tests/golden/preflop_ref.json) must give the same matrices within 2e-6: both
count wins and ties exactly and sum in the same order; the reference's
fast-math divisions (the equity and the class average) round within a few
ulps of IEEE division."""
import os

import numpy as np
import pytest

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_pf_flop_mats.npz")


@pytest.mark.parametrize("k", [0, 1, 2])
def test_class_matrix_matches_reference_kernels(orc, k):
    if not os.path.isfile(FIX):
        pytest.skip("tests/golden/ref_pf_flop_mats.npz not generated")
    z = np.load(FIX)
    ref = z["class_mats"][k]
    got = orc.pf_flop_class(z["flops"][k])
    assert got.shape == ref.shape == (169, 169)
    assert np.abs(got - ref).max() <= 2e-6
    assert np.mean(got.view(np.uint32) == ref.view(np.uint32)) > 0.5
