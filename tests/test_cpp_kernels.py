"""The C++ kernel classes (include/interax_b200_kernels.hpp) driven like a platform would drive them: built with g++
against the library, fed a water box through Force objects with the reference's accessors, checked against the
Python Context (the same C ABI underneath, so the results are identical)."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from interaxplugin import workloads as W

ROOT = Path(__file__).resolve().parent.parent
LIBDIR = ROOT / "openmm-interax-plugin_b200"


def build(tmp_path):
    exe = tmp_path / "kernels_from_file"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/kernels_from_file.cpp"),
           "-L", str(LIBDIR), "-linterax_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)]
    subprocess.run(cmd, check=True)
    return exe


def write_system(path, system, pos, box, lam=1.0):
    n = system.getNumParticles()
    out = [str(n), " ".join(repr(float(x)) for x in np.asarray(box).reshape(9)), repr(lam),
           " ".join(repr(float(x)) for x in np.asarray(pos).reshape(-1))]
    for t in range(3):
        f = system.getForce(t)
        head = [f.getNonbondedMethod(), f.getCutoffDistance(), int(f.getUseSwitchingFunction()),
                f.getSwitchingDistance(), f.getSoftcoreRadius(), f.getForceGroup()]
        head += [f.getDampingScale(), int(f.getUseLongRangeCorrection())] if t == 0 else [f.getOverlapMethod()]
        ex = np.asarray(f._exclusion_array()).reshape(-1)
        out += [" ".join(repr(x) for x in head), " ".join(repr(float(x)) for x in np.asarray(f._params_array()).reshape(-1)),
                " ".join(str(int(a)) for a in f._alch_array()), str(len(ex) // 2), " ".join(str(int(x)) for x in ex)]
    atm = system.getForce(3)
    off, part, params, mol, alch = atm._site_arrays()
    out.append(" ".join(repr(x) for x in [atm.getNumSites(), atm.getCutoffDistance(), atm.getScaleFactor(),
                                         atm.getDampingMethod(), atm.getDampingScale(),
                                         atm.getCentroidDampingRadius(), int(atm.usesPeriodicBoundaryConditions()),
                                         atm.getForceGroup()]))
    params = np.asarray(params).reshape(-1, 3)
    for s in range(atm.getNumSites()):
        p = part[off[s]:off[s + 1]]
        out.append(" ".join([str(len(p))] + [str(int(q)) for q in p] + [repr(float(v)) for v in params[s]] +
                            [str(int(mol[s])), str(int(alch[s]))]))
    path.write_text("\n".join(out) + "\n")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_header_compiles_and_reports_missing_device(tmp_path):
    """Without a GPU the shared context throws, with the library's message."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; test_cpp_kernels_match_context covers this machine")
    exe = build(tmp_path)
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=1,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    write_system(tmp_path / "in.txt", system, pos, box)
    r = subprocess.run([str(exe), str(tmp_path / "in.txt"), str(tmp_path / "out.txt")], capture_output=True, text=True)
    assert r.returncode == 1
    assert "error:" in r.stderr and ("device" in r.stderr or "CUDA" in r.stderr)


@pytest.mark.gpu
def test_cpp_kernels_match_context(tmp_path):
    from interaxplugin import Context
    exe = build(tmp_path)
    cfg = W.CONFIGS["small"]
    system, pos, box = W.water_box(cfg["num_waters"], cfg["box_length"], cfg["cutoff"], seed=11,
                                   three_body_cutoff=cfg["three_body_cutoff"])
    write_system(tmp_path / "in.txt", system, pos, box)
    subprocess.run([str(exe), str(tmp_path / "in.txt"), str(tmp_path / "out.txt")], check=True)
    lines = (tmp_path / "out.txt").read_text().splitlines()
    energies = np.array([float(x) for x in lines[0].split()])
    n = system.getNumParticles()
    forces = np.array([float(x) for x in lines[1:1 + 3 * n]]).reshape(n, 3)
    assert lines[1 + 3 * n].startswith("factory: Tried to create kernel with illegal kernel name")
    ctx = Context(system)
    ctx.setPeriodicBoxVectors(*np.asarray(box))
    ctx.setPositions(pos)
    st = ctx.getState()
    assert np.array_equal(energies, st.getTermEnergies())
    assert np.array_equal(forces, st.getForces())
