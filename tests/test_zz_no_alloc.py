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


def _cluster_call(num_waters, seed, stream, d=None):
    """ix_three_body_noalloc on a water cluster with no three-body cutoff (site a has every later site as a
    neighbor), and the context's own three-body result.  Returns the call, the reference and the device buffers."""
    import torch
    system, pos, _ = W.water_cluster(num_waters, seed=seed)
    atm = system.getForce(3)
    ctx = Context(system)
    ctx.setPositions(pos)
    st = ctx.getState(groups=1 << atm.getForceGroup())
    off, part, params, mol, alch = atm._site_arrays()
    dev = torch.device("cuda:0")
    if d is None:
        d = dict(pos=torch.tensor(pos, dtype=torch.float64, device=dev),
                 off=torch.tensor(off, dtype=torch.int32, device=dev),
                 part=torch.tensor(part, dtype=torch.int32, device=dev),
                 params=torch.tensor(params, dtype=torch.float64, device=dev),
                 mol=torch.tensor(mol, dtype=torch.int32, device=dev),
                 alch=torch.tensor(alch, dtype=torch.uint8, device=dev),
                 forces=torch.zeros((len(pos), 3), dtype=torch.float64, device=dev),
                 energy=torch.zeros(1, dtype=torch.float64, device=dev))
    L = _capi.lib()

    def call():
        return L.ix_three_body_noalloc(len(pos), _ptr(d["pos"]), None, atm.getNumSites(), _ptr(d["off"]),
                                       _ptr(d["part"]), _ptr(d["params"]), _ptr(d["mol"]), _ptr(d["alch"]),
                                       atm.getCutoffDistance(), atm.getScaleFactor(), atm.getDampingMethod(),
                                       atm.getDampingScale(), atm.getCentroidDampingRadius(), 0, 1.0,
                                       _ptr(d["forces"]), _ptr(d["energy"]), ctypes.c_void_p(stream.cuda_stream))
    return call, (st.getPotentialEnergy(), st.getForces()), d


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _overflow():
    L = _capi.lib()
    flag = ctypes.c_int(-1)
    assert L.ix_three_body_noalloc_overflow(ctypes.byref(flag)) == 0
    return flag.value


@pytest.mark.parametrize("num_waters,overflow", [(110, 0), (170, 1)])
def test_noalloc_long_and_overflowing_lists(num_waters, overflow):
    """110 waters: the first sites have 65 to 109 later neighbors (the long-list kernel, within the 128-entry lists);
    170 waters: the first 41 sites have more than 128 and are evaluated by a scan of every later site, which the
    overflow query reports.  The call runs on a non-blocking stream and the query is made without synchronizing
    first: the query itself waits for the device."""
    import torch
    stream = torch.cuda.Stream()
    call, (e_ref, f_ref), d = _cluster_call(num_waters, 31, stream)
    torch.cuda.synchronize()
    for repeat in range(2):
        with torch.cuda.stream(stream):
            d["forces"].fill_(99.0)
        assert call() == 0, _capi.lib().ix_last_error(None).decode()
        assert _overflow() == overflow
        e_err, f_err = errors(float(d["energy"].item()), d["forces"].cpu().numpy(), e_ref, f_ref)
        assert e_err <= 1e-6 and f_err <= 1e-5, (repeat, e_err, f_err)


def test_noalloc_captured_in_a_cuda_graph():
    """A call captured into a CUDA graph on a torch stream (after a first call outside capture, which looks up the
    scratch address), replayed twice: the second replay after the positions were moved in place, against the
    context's result at each set of positions."""
    import torch
    stream = torch.cuda.Stream()
    call, (e0, f0), d = _cluster_call(40, 33, stream)
    with torch.cuda.stream(stream):
        assert call() == 0
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        assert call() == 0
    system, pos, _ = W.water_cluster(40, seed=33)
    moved = pos + 0.01 * np.sin(np.arange(pos.size)).reshape(pos.shape)
    atm = system.getForce(3)
    ctx = Context(system)
    ctx.setPositions(moved)
    st = ctx.getState(groups=1 << atm.getForceGroup())
    for positions, (e_ref, f_ref) in ((pos, (e0, f0)), (moved, (st.getPotentialEnergy(), st.getForces()))):
        d["pos"].copy_(torch.tensor(positions, dtype=torch.float64))
        d["forces"].fill_(-1.0)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        e_err, f_err = errors(float(d["energy"].item()), d["forces"].cpu().numpy(), e_ref, f_ref)
        assert e_err <= 1e-6 and f_err <= 1e-5, (e_err, f_err)
    del graph


def test_noalloc_rejects_sizes_beyond_the_limit():
    L = _capi.lib()
    dummy = ctypes.c_void_p(1)
    rc = L.ix_three_body_noalloc(16385, dummy, None, 3, dummy, dummy, dummy, dummy, dummy, 1.0, 1.0, 0, 1.0, 0.0, 0,
                                 1.0, dummy, dummy, None)
    assert rc != 0 and b"limit is 16384" in L.ix_last_error(None)
    rc = L.ix_three_body_noalloc(10, dummy, None, 4097, dummy, dummy, dummy, dummy, dummy, 1.0, 1.0, 0, 1.0, 0.0, 0,
                                 1.0, dummy, dummy, None)
    assert rc != 0 and b"limit is 4096" in L.ix_last_error(None)
