"""Drop-in for the reference's HornSchunck module (src/HornSchunck.py).

HS runs on the GPU (of_hs_solve): 2x2-cube derivatives and `Niter` Jacobi sweeps,
bit-exact with the reference's scipy/numba float32 fields.
"""
import numpy as np

from ofb200 import ops, to_device, is_host, to_host, _torch

__all__ = ["HSOpticalFlowAlgoAdapter", "HS", "computeDerivatives"]


class HSOpticalFlowAlgoAdapter(object):
    """src/HornSchunck.py:28-49.  `alphas` is popped from the end, one per compute()."""

    def __init__(self, alphas, Niter, provideGenericPyramidalDefaults=True):
        self.provideGenericPyramidalDefaults = provideGenericPyramidalDefaults
        self.alphas = alphas
        self.Niter = Niter

    def compute(self, im1, im2, U, V):
        alpha = self.alphas.pop()  # Remove last alpha from the list
        return HS(im1, im2, alpha, self.Niter, U, V)

    def _compute_dev(self, im1, im2, U, V):
        """Device path used by the pyramid driver: no host synchronisation; the error is a
        device float64 scalar."""
        alpha = self.alphas.pop()
        U, V = U.clone(), V.clone()
        return ops.hs_solve(im1, im2, U, V, alpha, self.Niter)

    # CUDA-graph support (ofb200.graph): the key holds the alphas the next `n` calls pop
    def _graph_key(self, n):
        if len(self.alphas) < n:
            raise IndexError('pop from empty list')
        return ("HS", int(self.Niter), tuple(float(a) for a in self.alphas[len(self.alphas) - n:]))

    def _graph_clone(self, n):
        return HSOpticalFlowAlgoAdapter(list(self.alphas), self.Niter, self.provideGenericPyramidalDefaults)

    def _graph_consume(self, n):
        for _ in range(n):
            self.alphas.pop()

    def getAlgoName(self):
        return 'Horn-Schunck'

    def hasGenericPyramidalDefaults(self):
        return self.provideGenericPyramidalDefaults

    def getGenericPyramidalDefaults(self):
        return {'warping': True, 'biLinear': True, 'scaling': True}


def HS(im2, im1, alpha, Niter, U, V):
    """src/HornSchunck.py:72-104 (argument names as in the reference: the first argument is
    the frame at t0).  Returns (U, V, total_error) with a float error."""
    host = is_host(im2)
    I0, I1 = to_device(im2), to_device(im1)
    Ud = to_device(U).clone()
    Vd = to_device(V).clone()
    Ud, Vd, err = ops.hs_solve(I0, I1, Ud, Vd, alpha, Niter)
    e = float(err.item())
    if host:
        return to_host(Ud), to_host(Vd), e
    return Ud, Vd, e


def computeDerivatives(im1, im2):
    """src/HornSchunck.py:106-126: fx, fy, ft of the 2x2 cube (scipy 'mirror' borders).
    HS() calls it as computeDerivatives(frame_t1, frame_t0)."""
    host = is_host(im1)
    fx, fy, ft = ops.hs_derivatives(to_device(im2), to_device(im1))
    if host:
        return to_host(fx), to_host(fy), to_host(ft)
    return fx, fy, ft
