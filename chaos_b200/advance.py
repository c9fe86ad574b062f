"""`advance_ensemble` (src/Integrators/ensemble.jl:24-45) on the B200: `n` steps of size tau of an integrator on the
Henon-Heiles flow from every start, one orbit per thread, states only. The device work is
`cl_b200_advance_ensemble` (chaos_b200/csrc/cl_advance.cu); this is the host side: the reference's argument handling
(`chunk` as in the reference: None = all orbits per launch, else at least 1) and the (states, ok) result."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._lib import last_error, lib
from .foundation import DeviceError
from .systems import CorrectedMethod, Gauss, HenonHeilesFlow, IntegratorMap, SplittingMethod


def advance_ensemble(m, flow, x0, tau: float, n: int, *, chunk: int | None = None):
    """(states (len, 4), ok (len,) bool): `n` steps of size `tau` of `m` (a SplittingMethod, advanced by advance_n
    with kicks merged across the step boundary, or Gauss(3), advanced by advance_checked per step) on `flow`
    (HenonHeilesFlow) from every row of `x0`. `ok[j]` is False when an implicit step of orbit j failed; its state is
    then all NaN. The result of an orbit does not depend on `chunk`."""
    if not isinstance(m, (SplittingMethod, CorrectedMethod, Gauss)):
        raise TypeError("the compiled menu advances a SplittingMethod table, a CorrectedMethod or Gauss(3)")
    if not isinstance(flow, HenonHeilesFlow):
        raise TypeError("the compiled menu integrates HenonHeilesFlow")
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    if x0.ndim != 2 or x0.shape[1] != 4:
        raise ValueError("x0 must be an (orbits x 4) array of Henon-Heiles states")
    cs = IntegratorMap(m, flow, tau).to_cl()
    N = len(x0)
    csz = max(N, 1) if chunk is None else max(int(chunk), 1)
    out = np.empty_like(x0)
    ok = np.zeros(N, np.uint8)
    prov = _abi.cl_prov()
    rc = lib().cl_b200_advance_ensemble(C.byref(cs), N, x0.ctypes.data, out.ctypes.data, ok.ctypes.data,
                                        max(int(n), 0), csz, C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    return out, ok.astype(bool)
