"""Drop-in for the reference's denseLucasKanade_PyCL module
(src/denseLucasKanade_PyCL.py): dense pyramidal Lucas-Kanade on the GPU (of_lk_dense).

Same constructor and compute() as the OpenCL class; platformID is accepted and ignored,
deviceID selects the CUDA device.  compute() returns (U, V, True) like the reference.
The status / error planes the reference computes and discards are available through
compute_with_status().  The reference allocates its error buffer as uint8 while the kernel
writes float32 (:146 vs pyrlkDenseLargeW.cl:667); here it is a float32 plane.
"""
import numpy as np

from ofb200 import device_of, ops, to_device, is_host, to_host, _torch, log

__all__ = ["denseLucasKanade_PyCl"]


class denseLucasKanade_PyCl(object):
    def __init__(self, platformID=0, deviceID=0, Niter=5, halfWindow=13, provideGenericPyramidalDefaults=True,
                 enableVorticityEnhancement=False):
        self.provideGenericPyramidalDefaults = provideGenericPyramidalDefaults
        self.enableVorticityEnhancement = enableVorticityEnhancement
        self.device = device_of(platformID, deviceID)
        log('Running on device: ' + str(self.device))
        if not 1 <= halfWindow <= 15:
            raise ValueError("halfWindow must be in 1..15 (the kernel's 32x32 window grid)")
        self.windowHalfWidth = int(halfWindow)
        self.windowHalfHeight = int(halfWindow)
        self.windowWidth = 2 * halfWindow + 1
        self.windowHeight = 2 * halfWindow + 1
        self.Niter = Niter

    def evaluateVorticityEnhancement(self, U, V):
        """src/denseLucasKanade_PyCL.py:75-92: window masks from the sign of the mean
        vorticity (scipy 'reflect' borders)."""
        if not self.enableVorticityEnhancement:
            return [0, 0, 0, 0]
        torch = _torch()
        Ud, Vd = to_device(U), to_device(V)
        # D = [[0,-1,0],[0,0,0],[0,1,0]]*0.5; Dv = filter2(V, D.T, 'reflect'); Du = filter2(U, D, 'reflect')
        Vp = torch.cat([Vd[:, :1], Vd, Vd[:, -1:]], dim=1)
        Up = torch.cat([Ud[:1, :], Ud, Ud[-1:, :]], dim=0)
        Dv = (Vp[:, :-2].double() * 0.5 - Vp[:, 2:].double() * 0.5)
        Du = (Up[:-2, :].double() * 0.5 - Up[2:, :].double() * 0.5)
        m = float((Dv.float() - Du.float()).double().mean().item())
        if m < -2e-3:
            return [0, 1, 0, 1]
        if m > 2e-3:
            return [1, 0, 0, 1]
        return [0, 0, 0, 0]

    def calcPatchSize(self, windowWidth, windowHeight):
        if windowWidth > 32 and windowWidth > 2 * windowHeight:
            blockX, blockY = 32, 8
        else:
            blockX, blockY = 16, 16
        return np.int32((windowWidth + blockX - 1) / blockX), np.int32((windowHeight + blockY - 1) / blockY)

    def _run(self, im1, im2, U, V, want_status):
        torch = _torch()
        I, J = to_device(im1, self.device), to_device(im2, self.device)
        Ud, Vd = to_device(U, self.device).clone(), to_device(V, self.device).clone()
        asym = self.evaluateVorticityEnhancement(Ud, Vd)
        st = torch.empty(I.shape, dtype=torch.uint8, device=I.device) if want_status else None
        er = torch.empty(I.shape, dtype=torch.float32, device=I.device) if want_status else None
        ops.lk_dense(I, J, Ud, Vd, self.windowHalfWidth, self.Niter, asym, st, er)
        return Ud, Vd, st, er

    def _compute_dev(self, im1, im2, U, V):
        """compute() on device tensors; enqueues only (no host synchronisation) unless the
        vorticity enhancement has to read the mean vorticity back."""
        Ud, Vd, _, _ = self._run(im1, im2, U, V, False)
        return Ud, Vd, True

    def compute(self, im1, im2, U, V):
        Ud, Vd, _, _ = self._run(im1, im2, U, V, False)
        if is_host(im1):
            return to_host(Ud), to_host(Vd), True
        return Ud, Vd, True

    def compute_with_status(self, im1, im2, U, V):
        """(U, V, status uint8, err float32): 1 = tracked, 0 = singular / left the image."""
        Ud, Vd, st, er = self._run(im1, im2, U, V, True)
        if is_host(im1):
            return to_host(Ud), to_host(Vd), to_host(st), to_host(er)
        return Ud, Vd, st, er

    def _graph_key(self, n):
        if self.enableVorticityEnhancement:
            return None  # the window masks are chosen on the host from the current flow
        return ("LK", int(self.Niter), int(self.windowHalfWidth), str(self.device))

    def _graph_clone(self, n):
        return self

    def _graph_consume(self, n):
        pass

    def getAlgoName(self):
        return 'OpenCL Dense LK'

    def hasGenericPyramidalDefaults(self):
        return self.provideGenericPyramidalDefaults

    def getGenericPyramidalDefaults(self):
        return {'warping': False, 'intermediateScaling': True, 'scaling': False}
