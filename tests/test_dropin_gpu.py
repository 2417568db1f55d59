"""The drop-in `fluam data.main` driver on the GPU: same keywords, same output
files and formats as src/saveParticles.cu, trajectories equal to the oracle's
within the FP32 tolerance."""
import os
import subprocess

import numpy as np
import pytest

from helpers import chains, rel_inf

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FLUAM = os.path.join(ROOT, "fluam_b200", "fluam")


def read_particles(path):
    """Parse a .particles / .velocityParticles file: {time: (3, np)}."""
    with open(path) as f:
        head = f.readline()
        assert head.startswith("#NUMBER PARTICLES ")
        n = int(head.split()[2])
        out = {}
        while True:
            line = f.readline()
            if not line:
                break
            t = float(line)
            rows = [f.readline().split() for _ in range(n)]
            out[t] = np.array(rows, dtype=float).T
    return n, out


def run_fluam(tmp_path, text):
    p = tmp_path / "data.main"
    p.write_text(text)
    r = subprocess.run([FLUAM, str(p)], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    # the reference's main() returns 1 on success (src/main.cpp:111)
    assert r.returncode == 1, r.stdout + r.stderr
    return r


def test_reference_style_input(tmp_path, oracle):
    out = tmp_path / "run"
    text = f"""# reference keywords only
stokesLimit
particles 1
numberparticles 27
cutoff 2.2449240966
maxNumberPartInCellNonBonded 20
maxNumberPartInCell 20
densfluid 1
shearviscosity 1
temperature 0.1
cells 32 32 32
celldimension 64 64 64
initfluid 1
backgroundvelocity 0 0 0
seed 12
numstepsRelaxation 0
numsteps 6
samplefreq 3
savefreq 0
dt 0.25
outputname {out}
"""
    r = run_fluam(tmp_path, text)
    assert "Stokes Limit  3" in r.stdout and "Stokes Limit  6" in r.stdout
    for ext in (".data.main", ".cuda", ".seed", ".time", ".particles", ".velocityParticles"):
        assert os.path.exists(str(out) + ext), ext
    assert open(str(out) + ".seed").read() == "12\n"
    assert open(str(out) + ".data.main").read().startswith("# reference keywords only\nstokesLimit\n")
    n, pos = read_particles(str(out) + ".particles")
    _, frc = read_particles(str(out) + ".velocityParticles")
    assert n == 27 and sorted(pos) == [0.75, 1.5] and sorted(frc) == [0.75, 1.5]
    # simple-cubic start (src/simpleCubic.cpp): 3 x 3 x 3 lattice, spacing 64/3
    g = (np.arange(3) + 0.5) * 64 / 3 - 32
    q0 = np.stack(np.meshgrid(g, g, g, indexing="ij"))[::-1].reshape(3, -1)
    o = oracle.Oracle(32, 32, 32, 64.0, 64.0, 64.0, q0, eta=1, kT=0.1, dt=0.25,
                      cutoff=2.2449240966, kernel=3, pair=oracle.PAIR_TABLE_LJ, seed=12)
    o.step(3)
    assert rel_inf(pos[0.75] - q0, o.positions() - q0) < 1e-5
    o.step(3)
    assert rel_inf(pos[1.5] - q0, o.positions() - q0) < 1e-5
    # precision 15 text
    line = open(str(out) + ".particles").read().splitlines()[2]
    assert max(len(x.replace("-", "").replace(".", "")) for x in line.split()) <= 15


def test_extension_keywords_coordinates_and_bonds(tmp_path, oracle):
    L = 32.0
    q, bi, bj = chains(8, 8, (L, L, L), 4)
    n = q.shape[1]
    coor = tmp_path / "start.coor"
    with open(coor, "w") as f:
        f.write(f"{n}\n")
        for i in range(n):
            f.write("%.17g %.17g %.17g\n" % (q[0, i], q[1, i], q[2, i]))
    bonds = tmp_path / "bonds.dat"
    with open(bonds, "w") as f:
        f.write(f"{len(bi)}\n")
        for a, b in zip(bi, bj):
            f.write(f"{a} {b} 10 1\n")
        f.write("1\n0 2.0 0 0.0 0.0 0.0\n")
    out = tmp_path / "chains"
    text = f"""stokesLimit
loadparticles 1
coordinates {coor}
bondedForces {bonds}
cutoff 1.5
shearviscosity 1
temperature 0.01
cells 32 32 32
celldimension 32 32 32
seed 5
numstepsRelaxation 2
numsteps 4
samplefreq 2
dt 0.005
outputname {out}
kernelPoints 4
pairPotential soft
softEpsilon 1.0
"""
    run_fluam(tmp_path, text)
    _, pos = read_particles(str(out) + ".particles")
    assert sorted(pos) == [0.01, 0.02]
    o = oracle.Oracle(32, 32, 32, L, L, L, q, eta=1, kT=0.01, dt=0.005, cutoff=1.5, kernel=4,
                      pair=oracle.PAIR_SOFT, seed=5)
    o.set_bonds(bi, bj, np.full(len(bi), 10.0), np.ones(len(bi)), fi=[0], fk=[2.0], fr0=[0.0],
                fxyz=[[0.0, 0.0, 0.0]])
    o.step(4)  # 2 relaxation steps + 2
    assert rel_inf(pos[0.01] - q, o.positions() - q) < 1e-5
    o.step(2)
    assert rel_inf(pos[0.02] - q, o.positions() - q) < 1e-5


@pytest.mark.parametrize("name", __import__("golden_cases").cases())
def test_golden_cases_against_reference_outputs(tmp_path, name):
    """The drop-in run on the inputs of each golden case reproduces the
    reference's own outputs (tests/golden) within the FP32 tolerance."""
    import shutil
    import golden_cases as G
    c = G.load(name)
    for f in os.listdir(c["dir"]):
        if not f.startswith("out."):
            shutil.copy(os.path.join(c["dir"], f), tmp_path / f)
    r = subprocess.run([FLUAM, "data.main"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 1, r.stdout + r.stderr
    _, pos = G.read_particles(str(tmp_path / "out.particles"))
    fv = tmp_path / "out.velocityParticles"
    ref_fv = os.path.join(c["dir"], "out.velocityParticles")
    assert fv.exists() == os.path.exists(ref_fv)
    frc = G.read_particles(str(fv))[1] if fv.exists() and c["frc"] is not None else None
    assert sorted(pos) == sorted(c["pos"])
    # the quasi-2D family is FP64 on the GPU, as the reference
    tol = 1e-9 if c["cfg"].scheme >= 2 else 1e-5
    for t in c["pos"]:
        assert rel_inf(pos[t] - c["q0"], c["pos"][t] - c["q0"]) < tol, (name, t)
        if frc is not None:
            assert np.abs(frc[t] - c["frc"][t]).max() <= 1e-5 * max(np.abs(c["frc"][t]).max(), 1e-300)
    if c["cfg"].scheme >= 2 and fv.exists():
        # stokesLimit2D's particle velocity array is never set: zeros, byte for byte
        assert fv.read_text() == open(ref_fv).read()


def test_errors_are_reported(tmp_path):
    p = tmp_path / "data.main"
    p.write_text("stokesLimit\ncells 8 8 8\nsamplefreq 0\noutputname x\n")
    r = subprocess.run([FLUAM, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0 and "samplefreq" in r.stdout
    # a scheme this build does not run
    p.write_text("incompressibleBinaryMixture\ncells 8 8 8\nsamplefreq 1\noutputname x\n")
    r = subprocess.run([FLUAM, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0 and "stokesLimit" in r.stdout
    # the incompressible scheme needs a density and rejects particles
    p.write_text("incompressible\ncells 8 8 8\nsamplefreq 1\noutputname x\n")
    r = subprocess.run([FLUAM, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0 and "densfluid" in r.stdout
    p.write_text("incompressible\nparticles 1\ndensfluid 1\ncells 8 8 8\nsamplefreq 1\noutputname x\n")
    r = subprocess.run([FLUAM, str(p)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0 and "incompressibleBoundary" in r.stdout


def test_fluid_output_files(tmp_path, fsl):
    """saveFluid 1 / saveVTK 1 / savefreq: <out>.fluidFinalConfiguration,
    snapshots <out>.<step/savefreq>.fluid.vtk at sample steps and the final
    <out>.fluid.vtk, holding the velocity field of the last solve."""
    out = tmp_path / "run"
    text = f"""stokesLimit
particles 1
numberparticles 27
cutoff 1.5
pairPotential soft
densfluid 1
shearviscosity 1
temperature 0.01
cells 16 16 16
celldimension 16 16 16
seed 3
numsteps 4
samplefreq 2
savefreq 2
saveFluid 1
saveVTK 1
dt 0.01
outputname {out}
"""
    run_fluam(tmp_path, text)
    for name in ("run.1.fluid.vtk", "run.2.fluid.vtk", "run.fluid.vtk", "run.fluidFinalConfiguration"):
        assert (tmp_path / name).exists(), name
    lines = (tmp_path / "run.fluidFinalConfiguration").read_text().split("\n")
    assert lines[0] == "Number of cells 4096" and lines[2] == "16 16 16"
    v_file = np.array([lines[13 + 2 * i].split() for i in range(4096)], dtype=float).T
    # the same run through the API: same seed, same steps, same bits
    c, run = fsl.parse_data_main(tmp_path / "data.main")
    g3 = (np.arange(3) + 0.5) * (16.0 / 3) - 16.0 / 2  # src/simpleCubic.cpp arithmetic
    q0 = np.stack(np.meshgrid(g3, g3, g3, indexing="ij"))[::-1].reshape(3, -1)
    sim = fsl.StokesLimit(c, q0)
    sim.step(4)
    v_api = sim.velocity64().reshape(3, -1)
    sim.close()
    assert np.allclose(v_file, v_api, rtol=1e-13, atol=1e-300)
    vtk = (tmp_path / "run.fluid.vtk").read_text()
    assert vtk.startswith("# vtk DataFile Version 2.0\nWritten using VisIt writer\nASCII\n")
    assert "DIMENSIONS 17 17 17" in vtk and "CELL_DATA 4096" in vtk
