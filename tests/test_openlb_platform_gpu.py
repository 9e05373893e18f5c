"""OpenLB's own example, unmodified, on Platform::GPU_B200.

examples/laminar/cavity3dBenchmark/cavity3d.cpp is compiled from its original
source by openlb_b200/platform/Makefile, in both of its set-ups (bb:
LID_DRIVEN_BOUNCE_BACK, bounce-back walls and a moving-wall lid; local: the
default, boundary::set<LocalVelocity> on walls and lid, whose box edges and
corners get OpenLB's outer edge and corner post-processors), twice each:
against OpenLB patched with the
GPU_B200 platform tag (PLATFORMS := CPU_SISD GPU_B200, so the load balancer
hands every cuboid to the B200 platform and each collideAndStream is one fused
device step through the C ABI) and as the plain CPU_SISD build.  Both run the
same command line; the example writes its physical velocity and pressure
(SuperLatticePhysVelocity3D / PhysPressure3D through SuperVTMwriter3D) after
the timed steps, and the two outputs must agree.

Tolerance: T = float in the example, and the lid-driven cavity amplifies
rounding: OpenLB's own CPU_SISD build with its CSE collision and the same
build with -DDISABLE_CSE (generic operation order) already differ by about
6e-5 of the lid speed in velocity after 110 steps at size 32.  The B200 run
must stay within twice that spread of the CSE build, in velocity and in
pressure; the spread itself is measured by the test from the two CPU builds.
"""
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.olb_vtk import read_vti

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parents[1] / "openlb_b200" / "platform" / "_bin"
SIZE, STEPS = 32, 100   # the example runs 10 warm-up steps before STEPS timed ones


def _run(binary: str, workdir: Path, *args, env=None):
    exe = BIN / binary
    assert exe.exists(), f"{exe} missing: build it with make -C openlb_b200/platform"
    r = subprocess.run([str(exe), *map(str, args)], cwd=workdir, capture_output=True, text=True,
                       timeout=600, env=dict(os.environ, **(env or {})))
    assert r.returncode == 0, f"{binary} failed ({r.returncode}): {r.stdout[-1500:]} {r.stderr[-1500:]}"
    return r.stdout


def _mlups(stdout: str) -> float:
    # the example's own last line: size, steps, cuboids, ranks, threads, MLUPs
    line = [l for l in stdout.splitlines() if re.match(r"^\d+, \d+, \d+, \d+, \d+, ", l)][-1]
    return float(line.split(",")[-1])


def _fields(workdir: Path):
    data = workdir / "tmp" / "vtkData" / "data"
    u = read_vti(data / "physVelocity_iT0000000iC00000.vti")["physVelocity"]
    p = read_vti(data / "physPressure_iT0000000iC00000.vti")["physPressure"]
    return u.astype(np.float64), p.astype(np.float64)


@pytest.mark.parametrize("variant", ["bb", "local"])
def test_cavity3d_example_on_gpu_b200_matches_cpu_sisd(tmp_path, variant):
    dirs = {k: tmp_path / k for k in ("sisd", "nocse", "b200")}
    for d in dirs.values():
        d.mkdir()
    out_sisd = _run(f"cavity3d_{variant}_sisd", dirs["sisd"], "--size", SIZE, "--steps", STEPS)
    _run(f"cavity3d_{variant}_sisd_nocse", dirs["nocse"], "--size", SIZE, "--steps", STEPS)
    out_b200 = _run(f"cavity3d_{variant}_b200", dirs["b200"], "--size", SIZE, "--steps", STEPS)
    assert _mlups(out_sisd) > 0 and _mlups(out_b200) > 0
    u_ref, p_ref = _fields(dirs["sisd"])
    u_gen, p_gen = _fields(dirs["nocse"])
    u, p = _fields(dirs["b200"])
    assert u.shape == u_ref.shape and p.shape == p_ref.shape
    lid = np.abs(u_ref).max()
    assert lid > 0.5   # the lid moves the fluid (physical lid speed 1)
    # the flow developed: interior velocities well above the tolerance
    inner = u_ref[2:-2, 2:-3, 2:-2]
    assert np.abs(inner).max() > 1e-2 * lid
    du = float(np.abs(u - u_ref).max())
    dp = float(np.abs(p - p_ref).max())
    du_own = float(np.abs(u_gen - u_ref).max())
    dp_own = float(np.abs(p_gen - p_ref).max())
    print(f"cavity3d {variant} size {SIZE}: max |du| {du:.3e} (OpenLB CSE vs generic {du_own:.3e}, lid {lid:.3f}), "
          f"max |dp| {dp:.3e} (OpenLB {dp_own:.3e}, range {np.ptp(p_ref):.3e}); "
          f"MLUPS sisd {_mlups(out_sisd):.1f} b200 {_mlups(out_b200):.1f}")
    assert 0 < du_own < 1e-3 * lid
    assert du <= 2 * du_own
    assert dp <= 2 * dp_own


@pytest.mark.parametrize("variant", ["bb", "local"])
def test_cavity3d_example_reports_device_throughput(tmp_path, variant):
    """The example's own timer (util::Timer, wall clock) over 200 steps of a
    128^3 cavity: with at most two steps in flight it measures the device."""
    out = _run(f"cavity3d_{variant}_b200", tmp_path, "--size", 128, "--steps", 200, "--no-results")
    assert _mlups(out) > 1000
