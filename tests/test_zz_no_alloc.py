"""The allocation-free three-body entry point, ix_three_body_noalloc.

It serves callers that cannot allocate device memory where they need forces (inside a CUDA graph capture, engines
that own all device memory through their own pool, step loops that must not allocate); its working memory is one
fixed __device__ array shared by every call.  This test calls it through the C ABI on device buffers and compares it,
on two calls in a row (the second call finds the previous call's contents in the shared array), with the context's
own three-body evaluation (ix_compute), within the tolerances of the other parity tests.

The file name sorts last so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from interaxplugin import Context, _capi
from interaxplugin import workloads as W
from parity import errors

pytestmark = pytest.mark.gpu


def _system():
    cfg = W.CONFIGS["small"]
    return W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=21, three_body_cutoff=0.6)


def test_noalloc_matches_context_three_body():
    import torch
    system, pos, box = _system()
    atm = system.getForce(3)
    ctx = Context(system)
    ctx.setPositions(pos)
    st = ctx.getState(groups=1 << atm.getForceGroup())
    e_ref, f_ref = st.getPotentialEnergy(), st.getForces()

    off, part, params, mol, alch = atm._site_arrays()
    dev = torch.device("cuda:0")
    d_pos = torch.tensor(pos, dtype=torch.float64, device=dev)
    d_off = torch.tensor(off, dtype=torch.int32, device=dev)
    d_part = torch.tensor(part, dtype=torch.int32, device=dev)
    d_params = torch.tensor(params, dtype=torch.float64, device=dev)
    d_mol = torch.tensor(mol, dtype=torch.int32, device=dev)
    d_alch = torch.tensor(alch, dtype=torch.uint8, device=dev)
    d_forces = torch.zeros((len(pos), 3), dtype=torch.float64, device=dev)
    d_energy = torch.zeros(1, dtype=torch.float64, device=dev)
    box9 = np.ascontiguousarray(np.asarray(box, dtype=np.float64).reshape(9))
    L = _capi.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream

    def ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    for call in range(2):
        d_forces.fill_(123.0)   # the call must overwrite every output value
        rc = L.ix_three_body_noalloc(len(pos), ptr(d_pos), _capi.ptr(box9), atm.getNumSites(), ptr(d_off),
                                     ptr(d_part), ptr(d_params), ptr(d_mol), ptr(d_alch), atm.getCutoffDistance(),
                                     atm.getScaleFactor(), atm.getDampingMethod(), atm.getDampingScale(),
                                     atm.getCentroidDampingRadius(), int(atm.usesPeriodicBoundaryConditions()), 1.0,
                                     ptr(d_forces), ptr(d_energy), ctypes.c_void_p(stream))
        assert rc == 0, L.ix_last_error(None).decode()
        torch.cuda.synchronize()
        e = float(d_energy.item())
        f = d_forces.cpu().numpy()
        e_err, f_err = errors(e, f, e_ref, f_ref)
        assert e_err <= 1e-6 and f_err <= 1e-5, (call, e, e_ref, e_err, f_err)
        overflow = ctypes.c_int(1)
        assert L.ix_three_body_noalloc_overflow(ctypes.byref(overflow)) == 0
        assert overflow.value == 0


def test_noalloc_rejects_sizes_beyond_the_limit():
    L = _capi.lib()
    dummy = ctypes.c_void_p(1)
    rc = L.ix_three_body_noalloc(16385, dummy, None, 3, dummy, dummy, dummy, dummy, dummy, 1.0, 1.0, 0, 1.0, 0.0, 0,
                                 1.0, dummy, dummy, None)
    assert rc != 0 and b"limit is 16384" in L.ix_last_error(None)
    rc = L.ix_three_body_noalloc(10, dummy, None, 4097, dummy, dummy, dummy, dummy, dummy, 1.0, 1.0, 0, 1.0, 0.0, 0,
                                 1.0, dummy, dummy, None)
    assert rc != 0 and b"limit is 4096" in L.ix_last_error(None)
