"""The device entry points, which a GPU engine calls with its own device arrays (no host round trip):

* ix_compute_device: positions set on the context, forces ADDED to an int64 fixed-point buffer (scale 2^32, rows of
  `stride`), as OpenMM's CUDA platform accumulates them (platforms/common/src/kernels/interaxThreeBody.cc:644-652);
* ix_compute_device_f64: FP64 device positions in, FP64 device forces out;
* ix_compute_device_posq: the platform's own position array (float4, float4 + correction, or double4) in its slot
  order with its atom index, forces added at each particle's slot of its int64 buffer, the energy added to a device
  double, and a device status word for list overflows (what CalcInterax*ForceKernel::execute does on the CUDA
  platform, platforms/common/src/CommonInteraxKernels.cpp:251-259 and 631-646).

Each is compared with ix_compute on the same positions: bitwise where the positions are the same doubles (the forces
are the same fixed-point sums), and with ix_compute at the rounded positions where the format rounds them.
"""
import ctypes

import numpy as np
import pytest

from interaxplugin import Context, _capi
from interaxplugin import workloads as W

pytestmark = pytest.mark.gpu

SCALE = float(2 ** 32)


def _setup(seed=5, alchemical=False):
    cfg = W.CONFIGS["small"]
    kw = dict(alchemical_waters=range(6), softcore_radius=0.1) if alchemical else {}
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=seed,
                                   three_body_cutoff=cfg["three_body_cutoff"], **kw)
    return system, pos, box


def _reference(system, pos, parameters=None):
    ctx = Context(system)
    ctx.setPositions(pos)
    for k, v in (parameters or {}).items():
        ctx.setParameter(k, v)
    st = ctx.getState()
    return st.getTermEnergies().copy(), st.getForces().copy()


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _sync(ctx):
    ctx._check(_capi.lib().ix_synchronize(ctx._ctx))


def test_compute_device_fixed_point_adds_bitwise():
    import torch
    system, pos, _ = _setup()
    e_ref, f_ref = _reference(system, pos)
    n = len(pos)
    ctx = Context(system)
    ctx.setPositions(pos)
    stride = n + 37
    buf = torch.full((3 * stride,), 5, dtype=torch.int64, device="cuda")
    energies = torch.zeros(4, dtype=torch.float64, device="cuda")
    L = _capi.lib()
    torch.cuda.synchronize()
    for call in (1, 2):
        ctx._check(L.ix_compute_device(ctx._ctx, -1, _p(buf), stride, _p(energies)))
        _sync(ctx)
        got = buf.view(3, stride).cpu().numpy()
        assert np.all(got[:, n:] == 5)                   # the padding rows are untouched
        # each call adds the forces to what the buffer holds
        assert np.array_equal((got[:, :n].T - 5) / SCALE, call * f_ref)
        assert np.array_equal(energies.cpu().numpy(), e_ref)
        status = ctypes.c_int(-1)
        ctx._check(L.ix_get_device_status(ctx._ctx, ctypes.byref(status)))
        assert status.value == 0


def test_compute_device_f64_matches_compute():
    import torch
    system, pos, box = _setup(seed=6)
    e_ref, f_ref = _reference(system, pos)
    ctx = Context(system)
    ctx.setPositions(pos + 0.3)          # replaced by the device positions below
    d_pos = torch.tensor(pos, dtype=torch.float64, device="cuda")
    d_f = torch.full((len(pos), 3), 7.0, dtype=torch.float64, device="cuda")
    d_e = torch.zeros(4, dtype=torch.float64, device="cuda")
    box9 = _capi.arr(np.asarray(box).reshape(9), np.float64)
    torch.cuda.synchronize()
    L = _capi.lib()
    ctx._check(L.ix_compute_device_f64(ctx._ctx, -1, _p(d_pos), _capi.ptr(box9), _p(d_f), _p(d_e)))
    _sync(ctx)
    assert np.array_equal(d_f.cpu().numpy(), f_ref)
    assert np.array_equal(d_e.cpu().numpy(), e_ref)


def _posq_call(ctx, fmt, posq, corr, atom_index, box9, buf, stride, energy, status):
    L = _capi.lib()
    return L.ix_compute_device_posq(ctx._ctx, -1, fmt, _p(posq), _p(corr) if corr is not None else None,
                                    _p(atom_index), _capi.ptr(box9), _p(buf), stride, _p(energy), _p(status))


@pytest.mark.parametrize("fmt", [_capi.IX_POSQ_DOUBLE4, _capi.IX_POSQ_FLOAT4_CORRECTED, _capi.IX_POSQ_FLOAT4])
@pytest.mark.parametrize("alchemical", [False, True])
def test_compute_device_posq(fmt, alchemical):
    import torch
    system, pos, box = _setup(seed=7, alchemical=alchemical)
    params = {"lambda_sterics": 0.6} if alchemical else None
    n = len(pos)
    rng = np.random.default_rng(1)
    perm = rng.permutation(n).astype(np.int32)         # slot k holds particle perm[k]
    stride = (n + 31) // 32 * 32 + 32
    if fmt == _capi.IX_POSQ_DOUBLE4:
        q = np.zeros((stride, 4))
        q[:n, :3] = pos[perm]
        posq, corr, used = torch.tensor(q, device="cuda"), None, pos
    else:
        hi = pos.astype(np.float32)
        q = np.zeros((stride, 4), dtype=np.float32)
        q[:n, :3] = hi[perm]
        posq = torch.tensor(q, device="cuda")
        if fmt == _capi.IX_POSQ_FLOAT4_CORRECTED:
            c = np.zeros((stride, 4), dtype=np.float32)
            c[:n, :3] = (pos - hi.astype(np.float64)).astype(np.float32)[perm]
            corr = torch.tensor(c, device="cuda")
            used = hi.astype(np.float64) + (pos - hi.astype(np.float64)).astype(np.float32).astype(np.float64)
        else:
            corr, used = None, hi.astype(np.float64)
    e_ref, f_ref = _reference(system, used, params)
    ctx = Context(system)
    ctx.setPositions(pos)
    for k, v in (params or {}).items():
        ctx.setParameter(k, v)
    atom_index = torch.tensor(perm, device="cuda")
    buf = torch.zeros(3 * stride, dtype=torch.int64, device="cuda")
    energy = torch.full((1,), 1.5, dtype=torch.float64, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    box9 = _capi.arr(np.asarray(box).reshape(9), np.float64)
    torch.cuda.synchronize()
    for call in range(2):                              # the second call replays the captured graph
        buf.zero_()
        energy.fill_(1.5)
        torch.cuda.synchronize()
        ctx._check(_posq_call(ctx, fmt, posq, corr, atom_index, box9, buf, stride, energy, status))
        _sync(ctx)
        rows = buf.view(3, stride).cpu().numpy()[:, :n].T     # slot order
        f = np.empty_like(f_ref)
        f[perm] = rows / SCALE
        assert np.array_equal(f, f_ref), np.abs(f - f_ref).max()
        assert abs(float(energy.item()) - 1.5 - e_ref.sum()) <= 1e-12 * np.abs(e_ref).sum()
        assert int(status.item()) == 0


def test_compute_device_posq_reports_and_recovers_from_overflow():
    import torch
    system, pos, box = _setup(seed=8)
    e_ref, f_ref = _reference(system, pos)
    n = len(pos)
    ctx = Context(system)
    ctx.setListCapacity(8, 2)
    ctx.setPositions(pos)
    q = np.zeros((n, 4))
    q[:, :3] = pos
    posq = torch.tensor(q, device="cuda")
    atom_index = torch.arange(n, dtype=torch.int32, device="cuda")
    buf = torch.zeros(3 * n, dtype=torch.int64, device="cuda")
    energy = torch.zeros(1, dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    box9 = _capi.arr(np.asarray(box).reshape(9), np.float64)
    torch.cuda.synchronize()
    ctx._check(_posq_call(ctx, _capi.IX_POSQ_DOUBLE4, posq, None, atom_index, box9, buf, n, energy, status))
    _sync(ctx)
    assert int(status.item()) & 1                       # incomplete: the pair list overflowed
    host = ctypes.c_int(0)
    ctx._check(_capi.lib().ix_get_device_status(ctx._ctx, ctypes.byref(host)))
    assert host.value == int(status.item())
    buf.zero_()
    energy.zero_()
    torch.cuda.synchronize()
    ctx._check(_posq_call(ctx, _capi.IX_POSQ_DOUBLE4, posq, None, atom_index, box9, buf, n, energy, status))
    _sync(ctx)
    assert int(status.item()) == 0
    f = buf.view(3, n).cpu().numpy().T / SCALE
    assert np.abs(f - f_ref).max() <= 1e-6 * np.abs(f_ref).max()
    assert abs(float(energy.item()) - e_ref.sum()) <= 1e-6 * np.abs(e_ref).sum()


def test_compute_device_posq_rejects_bad_arguments():
    system, pos, _ = _setup(seed=9)
    ctx = Context(system)
    ctx.setPositions(pos)
    L = _capi.lib()
    dummy = ctypes.c_void_p(16)
    assert L.ix_compute_device_posq(ctx._ctx, -1, 7, dummy, None, None, None, dummy, len(pos), None, None) != 0
    assert b"format" in L.ix_last_error(ctx._ctx)
    assert L.ix_compute_device_posq(ctx._ctx, -1, _capi.IX_POSQ_FLOAT4_CORRECTED, dummy, None, None, None, dummy,
                                    len(pos), None, None) != 0
    assert L.ix_compute_device_posq(ctx._ctx, -1, _capi.IX_POSQ_DOUBLE4, dummy, None, None, None, dummy,
                                    len(pos) - 1, None, None) != 0
