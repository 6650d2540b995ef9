"""Drop-in for the reference's PhysicsBasedOpticalFlowLiuShen module
(src/PhysicsBasedOpticalFlowLiuShen.py).

The solver runs on the GPU (of_ls_solve_mode); sweeps stop on the reference's rule
(error <= 1e-8 or 60 sweeps) decided on the device.  Two arithmetics, chosen per adapter
(`arithmetic=`) or for the process (OFB_LS_ARITHMETIC):
  'fast'  (default) the sweep in float32 with fused multiply-adds: fields within float32
          rounding of the reference's, <= 1e-3 px of the algorithm's float64 answer;
  'exact' bit-exact with the reference's float32 fields (float64 stencil sums in the
          reference's order, as scipy computes them).

Deviation: the reference declares hasGenericPyramidalDefaults() without `self`
(:44), so calling it raises TypeError and the adapter cannot be a main adapter.  Here it is
a regular method returning False.
"""
import numpy as np

from ofb200 import ops, to_device, is_host, to_host, log

__all__ = ["LiuShenOpticalFlowAlgoAdapter", "generate_invmatrix", "physicsBasedOpticalFlowLiuShen"]

MAXNUM = 60
TOL = 1e-8


class LiuShenOpticalFlowAlgoAdapter(object):
    """src/PhysicsBasedOpticalFlowLiuShen.py:33-45."""

    def __init__(self, alpha, arithmetic=None):
        self.alpha = alpha
        self.arithmetic = ops.ls_arithmetic(arithmetic)
        self.last_iterations = self.last_error = None

    def compute(self, im1, im2, U, V):
        [resV, resU, error] = physicsBasedOpticalFlowLiuShen(im1, im2, self.alpha, V, U, self.arithmetic)
        return [resU, resV, error]

    def _compute_dev(self, im1, im2, U, V):
        """Device path (no synchronisation).  Returns (U, V, err) with device scalars; the
        sweep count of the last call is kept in self.last_iterations (device int32)."""
        U, V = U.clone(), V.clone()
        U, V, it, err = ops.ls_solve(im1, im2, U, V, self.alpha, MAXNUM, TOL, arithmetic=self.arithmetic)
        self.last_iterations, self.last_error = it, err
        return U, V, err

    def _graph_key(self, n):
        return ("LS", float(self.alpha), self.arithmetic)

    def _graph_clone(self, n):
        return LiuShenOpticalFlowAlgoAdapter(self.alpha, self.arithmetic)

    def _graph_consume(self, n):
        pass

    def getAlgoName(self):
        return 'Liu-Shen Physics based OF'

    def hasGenericPyramidalDefaults(self):
        log("LiuShenOpticalFlowAlgoAdapter.hasGenericPyramidalDefaults: the reference raises TypeError here")
        return False


def generate_invmatrix(im, h, dx):
    """B11, B12, B22 = inverse of the 2x2 per-pixel system (:47-73); dx must be 1."""
    if dx != 1:
        raise NotImplementedError("generate_invmatrix: only dx == 1 (the reference's only use)")
    host = is_host(im)
    I = to_device(im)
    c = ops.ls_coefficients(I, I.new_zeros(I.shape), h)
    out = (c[5], c[6], c[7])
    return tuple(to_host(t) for t in out) if host else out


def physicsBasedOpticalFlowLiuShen(im1, im2, h, U, V, arithmetic=None):
    """:82-158.  U is the row (y) component and V the column (x) component here (the
    adapter swaps); returns (u, v, error) in the same convention with a float error."""
    host = is_host(im1)
    I0, I1 = to_device(im1), to_device(im2)
    Vx = to_device(V).clone()   # column component
    Uy = to_device(U).clone()   # row component
    Vx, Uy, it, err = ops.ls_solve(I0, I1, Vx, Uy, h, MAXNUM, TOL, arithmetic=arithmetic)
    e = float(err.item())
    if host:
        return to_host(Uy), to_host(Vx), e
    return Uy, Vx, e
