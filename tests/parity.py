"""Helpers of the parity tests: run a System on the B200 Context and on the FP64 oracle and compare."""
import math

import numpy as np

import pyoracle
from interaxplugin import Context

# Tolerances of the target: total energy within 1e-6 relative, forces within 1e-5 relative RMS of the FP64 oracle.
ENERGY_TOL = 1e-6
FORCE_RMS_TOL = 1e-5


def gpu_state(system, positions, box=None, parameters=None, groups=0xFFFFFFFF, context=None):
    ctx = context or Context(system)
    if box is not None:
        ctx.setPeriodicBoxVectors(*np.asarray(box))
    ctx.setPositions(positions)
    for k, v in (parameters or {}).items():
        ctx.setParameter(k, v)
    st = ctx.getState(groups=groups)
    return st.getPotentialEnergy(), st.getForces(), ctx


def errors(e, f, e_ref, f_ref, abs_energy=None):
    """Relative energy error (relative to |E| or to the given scale) and relative RMS force error."""
    scale = abs(e_ref) if abs_energy is None else abs_energy
    e_err = abs(e - e_ref) / max(scale, 1e-300)
    rms = math.sqrt((f_ref ** 2).sum() / max(f_ref.size, 1))
    f_err = math.sqrt(((f - f_ref) ** 2).sum() / max(f_ref.size, 1)) / max(rms, 1e-300)
    return e_err, f_err


# Resolution of forces accumulated in 64-bit fixed point with scale 2^32: a sum of a few contributions is exact
# only to ~1e-9 whatever the magnitude, so component errors below this are not counted, as in the reference's
# assertForcesEqual on GPU platforms (tests/InteraxTestUtilities.h:95-135).
FORCE_RESOLUTION = 1e-8


def max_force_error(f, f_ref):
    """Largest component error beyond the fixed-point resolution, relative to the largest expected force
    (tests/InteraxTestUtilities.h:108-135)."""
    scale = np.sqrt((f_ref ** 2).sum(1)).max()
    return max(np.abs(f - f_ref).max() - FORCE_RESOLUTION, 0.0) / max(scale, 1e-300)


def compare(system, positions, box=None, parameters=None, groups=0xFFFFFFFF, energy_tol=ENERGY_TOL,
            force_tol=FORCE_RMS_TOL, abs_energy=None, context=None, scale="total"):
    """Compare with the oracle.  scale="total": energy error relative to |E|; scale="abs": relative to the sum of
    |pair and triple energies|, the error scale of the reference's own tests (tests/TestInteraxPairForce.h:134-142)."""
    absE = []
    e_ref, f_ref = pyoracle.evaluate(system, positions, box, parameters, groups, abs_energy=absE)
    if scale == "abs" and abs_energy is None:
        abs_energy = max(absE[0], abs(e_ref))
    e, f, ctx = gpu_state(system, positions, box, parameters, groups, context)
    e_err, f_err = errors(e, f, e_ref, f_ref, abs_energy)
    assert np.all(np.isfinite(f))
    assert e_err <= energy_tol, f"energy {e} vs oracle {e_ref}: relative error {e_err:.3e} > {energy_tol}"
    assert f_err <= force_tol, f"forces: relative RMS error {f_err:.3e} > {force_tol}"
    return e, f, e_ref, f_ref, ctx
