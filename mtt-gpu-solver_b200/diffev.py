"""Differentiable EV of fixed strategies, as a torch.autograd.Function.

Both players play sigma = softmax(logits) at every decision node, per hand.
The forward pass is one sweep of the batch on the GPU (mtt_batch_ev_grad):
reach down the tree, terminal values of both players, counterfactual values
back up, and the adjoint of the softmax at every node.  It returns the root EV
of player 0 in chips and keeps the gradients, which the backward pass only
scales by the incoming gradient.  dEV0/drange are the root counterfactual
values ([cfv0 | -cfv1]); the values follow kernel_evaluate_terminals and
kernel_backward_sweep (honest_multistreet_solver.cu:128-249) with card removal.

    mtt = importlib.import_module("mtt-gpu-solver_b200")
    dev = mtt.diffev.StrategyEV(subgames)                 # packs once
    logits = torch.randn(dev.total_rows, device="cuda", requires_grad=True)
    r0, r1 = full 1,326-vectors [n, 1326] (requires_grad as needed)
    ev = dev(logits, dev.pack_ranges(r0, r1))              # [n]
    ev.sum().backward()                                    # logits.grad, r0.grad, r1.grad
"""
import numpy as np

from . import RiverBatch


class _EVFunction:
    """Holder of the autograd.Function class, built on first use so that
    importing the package does not import torch."""
    fn = None

    @classmethod
    def get(cls):
        if cls.fn is None:
            import torch

            class EVFn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, logits, ranges, owner):
                    ev, g_r, g_l = owner.batch.ev_grad(logits.detach().contiguous(), ranges.detach().contiguous())
                    ctx.save_for_backward(g_r, g_l)
                    ctx.owner = owner
                    return ev

                @staticmethod
                def backward(ctx, grad_ev):
                    g_r, g_l = ctx.saved_tensors
                    o = ctx.owner
                    gl = g_l * grad_ev[o.seg_rows] if ctx.needs_input_grad[0] else None
                    gr = g_r * grad_ev[o.seg_range] if ctx.needs_input_grad[1] else None
                    return gl, gr, None

            cls.fn = EVFn
        return cls.fn


class StrategyEV:
    """A batch of river subgames for the differentiable EV.

    subgames: dicts as for RiverBatch.  total_rows / total_range: lengths of
    the packed logit and range tensors; seg_rows / seg_range: subgame index of
    every packed element (padding included)."""

    def __init__(self, subgames, device=None):
        import torch
        self.device = torch.device(device or "cuda")
        self.batch = RiverBatch(subgames)
        lay = self.batch.layout()
        self.n = self.batch.n
        self.total_rows, self.total_range = lay["total_rows"], lay["total_range"]
        self.rows_off, self.range_off = lay["rows_off"], lay["range_off"]
        seg_rows = np.zeros(self.total_rows, np.int64)
        seg_range = np.zeros(self.total_range, np.int64)
        idx_r = [[], []]          # packed range index of every (subgame, combo) pair, per player
        sub_r = [[], []]
        cmb_r = [[], []]
        for s in range(self.n):
            rows0, rows1, H0, H1 = self.batch.meta[s]
            Hp = [(H0 + 3) // 4 * 4, (H1 + 3) // 4 * 4]
            seg_rows[self.rows_off[s, 0]:self.rows_off[s, 0] + rows0 * Hp[0]] = s
            seg_rows[self.rows_off[s, 1]:self.rows_off[s, 1] + rows1 * Hp[1]] = s
            seg_range[self.range_off[s]:self.range_off[s] + Hp[0] + Hp[1]] = s
            for p in range(2):
                c = self.batch.combos[s][p]
                base = self.range_off[s] + (Hp[0] if p else 0)
                idx_r[p].append(base + np.arange(len(c)))
                sub_r[p].append(np.full(len(c), s))
                cmb_r[p].append(c)
        t = lambda a: torch.from_numpy(np.concatenate(a) if isinstance(a, list) else a).to(self.device)
        self.seg_rows, self.seg_range = t(seg_rows), t(seg_range)
        self._ridx = [t(idx_r[p]) for p in range(2)]
        self._rsub = [t(sub_r[p]) for p in range(2)]
        self._rcmb = [t(cmb_r[p]) for p in range(2)]

    def pack_ranges(self, r0, r1):
        """[n, 1326] range vectors (combo ids 0..1325) -> packed [total_range].
        Differentiable: gradients flow back to r0 / r1 at each subgame's combos."""
        import torch
        out = torch.zeros(self.total_range, dtype=torch.float32, device=self.device)
        for p, r in enumerate((r0, r1)):
            out = out.index_put((self._ridx[p],), r[self._rsub[p], self._rcmb[p]].float())
        return out

    def unpack_rows(self, packed, s):
        """Subgame s's part of a rows-layout tensor: ([rows0, H0], [rows1, H1])."""
        rows0, rows1, H0, H1 = self.batch.meta[s]
        Hp = [(H0 + 3) // 4 * 4, (H1 + 3) // 4 * 4]
        out = []
        for p, (rows, H) in enumerate(((rows0, H0), (rows1, H1))):
            o = int(self.rows_off[s, p])
            out.append(packed[o:o + rows * Hp[p]].view(rows, Hp[p])[:, :H])
        return out

    def __call__(self, logits, ranges):
        return _EVFunction.get().apply(logits, ranges, self)

    def close(self):
        self.batch.close()
