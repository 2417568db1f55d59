"""Generate the golden fixtures of tests/golden/ from the reference itself.

Each case is a data.main (plus coordinate and bond files) using only the
reference's own features (LJ force table, 3-point kernel, bonds, tethers,
extraMobility, the reference RFD).  It is run through oracle/_ref/fluam_ref,
the reference's stokesLimit sources compiled for the host by
oracle/ref_cpu/build_ref.py (cuFFT replaced by a direct DFT, cuRAND by the
Philox normals shared with the oracle and the CUDA path).  The script keeps
the inputs and the reference's .particles / .velocityParticles / .seed.

Usage (in a container where the reference sources are mounted):
    python oracle/ref_cpu/build_ref.py && python tests/golden/make_golden.py
"""
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FLUAM_REF = os.path.join(ROOT, "oracle", "_ref", "fluam_ref")

FIRST_ORDER = "stokesLimitFirstOrder\nstokesLimit"

COMMON = """stokesLimit
particles 1
maxNumberPartInCellNonBonded 40
maxNumberPartInCell 40
densfluid 1
initfluid 0
backgroundvelocity 0 0 0
outputname out
"""


def lattice(n_per_side, spacing, jitter, seed, origin):
    g = np.arange(n_per_side) * spacing
    q = np.stack(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1) + np.asarray(origin)[:, None]
    return q + np.random.default_rng(seed).uniform(-jitter, jitter, q.shape)


def chains(nch, beads, box, seed):
    rng = np.random.default_rng(seed)
    starts = rng.uniform(-0.5, 0.5, (nch, 3)) * np.asarray(box)
    d = rng.standard_normal((nch, beads - 1, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    pos = np.concatenate([starts[:, None, :], starts[:, None, :] + np.cumsum(d, axis=1)], axis=1)
    q = pos.reshape(-1, 3).T.copy()
    idx = np.arange(nch * beads).reshape(nch, beads)
    return q, list(zip(idx[:, :-1].ravel(), idx[:, 1:].ravel()))


def chains2d(nch, beads, box, seed):
    """Chains in the plane z = 0: seeded starts, unit bonds in random directions."""
    rng = np.random.default_rng(seed)
    starts = rng.uniform(-0.5, 0.5, (nch, 2)) * np.asarray(box[:2])
    # directions turn by at most 0.6 rad per bond, so a chain never folds back
    phi = rng.uniform(0, 2 * np.pi, (nch, 1)) + np.cumsum(rng.uniform(-0.6, 0.6, (nch, beads - 1)), axis=1)
    d = np.stack([np.cos(phi), np.sin(phi)], axis=2)
    pos = np.concatenate([starts[:, None, :], starts[:, None, :] + np.cumsum(d, axis=1)], axis=1)
    q = np.zeros((3, nch * beads))
    q[:2] = pos.reshape(-1, 2).T
    idx = np.arange(nch * beads).reshape(nch, beads)
    return q, list(zip(idx[:, :-1].ravel(), idx[:, 1:].ravel()))


def write_coor(path, q):
    with open(path, "w") as f:
        f.write(f"{q.shape[1]}\n")
        for i in range(q.shape[1]):
            f.write("%.17g %.17g %.17g\n" % tuple(q[:, i]))


CASES = {
    # simple-cubic start of src/simpleCubic.cpp, no particle overlaps
    "lattice27": dict(text="""numberparticles 27
cutoff 2.2449240966
shearviscosity 1
temperature 0.01
cells 16 16 16
celldimension 16 16 16
seed 3
numsteps 4
samplefreq 1
dt 0.01
"""),
    # LJ table forces active: jittered lattice just inside the WCA cutoff
    # (sigma = 2 dx = 1, rc = 2^(1/6) sigma)
    "lj_dense": dict(text="""loadparticles 1
coordinates start.coor
cutoff 1.12246204830937
shearviscosity 1.3
temperature 0.05
cells 32 32 32
celldimension 16 16 16
seed 11
numsteps 3
samplefreq 1
dt 0.001
""", coor=lambda: lattice(6, 1.05, 0.04, 5, (-2.6, -2.6, -2.6))),
    # chains + tethers, extraMobility, no pair forces, non-cubic grid and box
    "bonds_extra": dict(text="""loadparticles 1
coordinates start.coor
bondedForces bonds.dat
computeNonBondedForces 0
cutoff 1.5
extraMobility 0.2
shearviscosity 0.8
temperature 0.02
cells 16 24 32
celldimension 16 24 32
seed 21
numstepsRelaxation 2
numsteps 4
samplefreq 2
dt 0.01
""", chains=(6, 8, (16.0, 24.0, 32.0), 9)),
    # the old bond-file format (bondedForcesVersion 1,
    # src/initializeBondedForcesOldVersion.cpp): every bond listed from both
    # ends and sorted by the first index, two springs listed from one end
    # only (each pulls its own particle alone; an even line count, because
    # the reference copies 2 (count / 2) lines to the device,
    # src/createBondedForcesGPU.cu:62-78), one tether per particle (the
    # reference misplaces a particle's second tether in this format)
    "bonds_old_format": dict(old_bonds=True, text="""loadparticles 1
coordinates start.coor
bondedForces bonds.dat
bondedForcesVersion 1
computeNonBondedForces 0
cutoff 1.5
extraMobility 0.1
shearviscosity 1.2
temperature 0.02
cells 24 16 20
celldimension 24 16 20
seed 33
numstepsRelaxation 1
numsteps 4
samplefreq 2
dt 0.01
""", chains=(5, 7, (24.0, 16.0, 20.0), 15)),
    # the first-order scheme (keyword stokesLimitFirstOrder, which takes
    # precedence over stokesLimit, src/main.cpp:94-99) with LJ forces.  The
    # stokesLimit keyword stays in the file: without it the reference never
    # copies the cell-centre coordinates to the device
    # (src/initializeFluidIncompressibleGPU.cu:27 tests stokesLimit only) and
    # its first-order kernels read uninitialised memory
    "first_order_lj": dict(scheme=FIRST_ORDER, text="""loadparticles 1
coordinates start.coor
cutoff 1.12246204830937
shearviscosity 0.9
temperature 0.05
cells 24 24 24
celldimension 12 12 12
seed 13
numsteps 3
samplefreq 1
dt 0.001
""", coor=lambda: lattice(5, 1.05, 0.04, 7, (-2.1, -2.1, -2.1))),
    # first order with chains, tethers and extraMobility (forces at the
    # midpoint) on a non-cubic grid
    "first_order_extra": dict(scheme=FIRST_ORDER, text="""loadparticles 1
coordinates start.coor
bondedForces bonds.dat
computeNonBondedForces 0
cutoff 1.5
extraMobility 0.3
shearviscosity 1.1
temperature 0.02
cells 20 16 24
celldimension 20 16 24
seed 29
numstepsRelaxation 1
numsteps 4
samplefreq 2
dt 0.01
""", chains=(5, 7, (20.0, 16.0, 24.0), 12)),
    # the quasi-2D family (keywords quasi2D / stokesLimit2D, src/runSchemeQuasi2D.cu):
    # a Gaussian-blob RPY step with LJ forces through the 2-D cell list and
    # the thermal drift (lz >= cutoff keeps the reference's neighbour grid
    # non-empty, src/createBoundariesQuasi2DGPU.cu:89-95)
    "q2d_rpy_lattice": dict(scheme="quasi2D", text="""numberparticles 100
computeNonBondedForces 1
cutoff 2.2449240966
shearviscosity 1.2
temperature 0.05
hydrodynamicRadius 1.0
cells 24 24 1
celldimension 24 24 4
seed 31
numstepsRelaxation 1
numsteps 6
samplefreq 2
dt 0.01
"""),
    # predictor-corrector with 2-D bonded chains and tethers (bonds act only
    # with computeNonBondedForces 1 in this scheme; a fine grid keeps the
    # hard-coded LJ table, sigma = 2 dx, short of the unit bonds)
    "q2d_pc_chains": dict(scheme="quasi2D", dim=2, text="""loadparticles 1
coordinates start.coor
bondedForces bonds.dat
computeNonBondedForces 1
cutoff 0.5612310241
predictorCorrector 1
shearviscosity 0.8
temperature 0.02
hydrodynamicRadius 0.5
cells 40 40 1
celldimension 10 10 4
seed 37
numsteps 4
samplefreq 2
dt 0.01
""", chains=(4, 5, (10.0, 10.0, 4.0), 17)),
    # 2-D Stokes mobility, no thermal drift
    "s2d_spectral": dict(scheme="stokesLimit2D", text="""numberparticles 25
computeNonBondedForces 1
cutoff 2.2449240966
use_RFD 0
shearviscosity 0.9
temperature 0.1
hydrodynamicRadius 1.2
cells 30 20 1
celldimension 30 20 4
seed 41
numsteps 4
samplefreq 2
dt 0.02
"""),
    # Saffman-screened 2-D mobility with the periodic layer correction and
    # the shear forcing, predictor-corrector, no forces
    "s2d_saffman_shear": dict(scheme="stokesLimit2D", text="""saffmanCutOffWaveNumber 0.3
saffmanLayerWidth 2.0
viscosityMeasureAmplitude 0.05
numberparticles 16
computeNonBondedForces 0
cutoff 2.0
predictorCorrector 1
shearviscosity 1.0
temperature 0.1
hydrodynamicRadius 1.0
cells 32 32 1
celldimension 32 32 1
seed 43
numsteps 4
samplefreq 2
dt 0.05
"""),
    # the incompressible fluctuating fluid (keyword incompressible, no
    # particles): a uniform start, noise-driven with advection
    "inc_fluid": dict(scheme="incompressible", fluid_only=True, text="""densfluid 1.3
shearviscosity 0.7
temperature 0.5
cells 12 16 20
celldimension 12 16 20
initfluid 0
backgroundvelocity 0.1 -0.05 0.02
numstepsRelaxation 1
numsteps 4
samplefreq 2
dt 0.05
seed 3
"""),
    # a non-cubic box, stronger advection (large background flow)
    "inc_fluid_flow": dict(scheme="incompressible", fluid_only=True, text="""densfluid 0.8
shearviscosity 1.1
temperature 0.05
cells 16 10 14
celldimension 24 15 14
initfluid 0
backgroundvelocity 0.8 0.3 -0.4
numsteps 6
samplefreq 3
dt 0.1
seed 8
"""),
}


def make_case(name, spec):
    d = os.path.join(HERE, name)
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    with open(os.path.join(d, "data.main"), "w") as f:
        common = COMMON
        if "scheme" in spec:
            common = common.replace("stokesLimit\n", spec["scheme"] + "\n", 1)
        if spec.get("fluid_only"):  # a fluid without particles
            common = spec["scheme"] + "\noutputname out\n"
        f.write(common + spec["text"])
    if "coor" in spec:
        write_coor(os.path.join(d, "start.coor"), spec["coor"]())
    if "chains" in spec:
        nch, beads, box, seed = spec["chains"]
        q, bonds = (chains2d if spec.get("dim") == 2 else chains)(nch, beads, box, seed)
        write_coor(os.path.join(d, "start.coor"), q)
        with open(os.path.join(d, "bonds.dat"), "w") as f:
            if spec.get("old_bonds"):
                # each bond from both ends, sorted by the first index; the
                # last chain's first bead is pulled towards bead 2 of chain
                # 0, and bead 10 towards bead 30, by springs listed from one
                # end only
                ent = []
                for k, (a, b) in enumerate(bonds):
                    ks, r0 = (10.0 if k % 2 else 4.0), (1.0 if k % 3 else 0.0)
                    ent += [(a, b, ks, r0), (b, a, ks, r0)]
                ent.append((nch * beads - beads, 2, 3.0, 2.0))
                ent.append((10, 30, 2.5, 1.5))
                ent.sort(key=lambda e: e[0])
                f.write(f"{len(ent)}\n")
                for a, b, ks, r0 in ent:
                    f.write(f"{a} {b} {ks} {r0}\n")
                f.write("2\n0 2.0 0.0 0.0 0.0 0.0\n5 1.5 0.5 1.0 -2.0 3.0\n")
            else:
                f.write(f"{len(bonds)}\n")
                for k, (a, b) in enumerate(bonds):
                    f.write(f"{a} {b} {10.0 if k % 2 else 4.0} {1.0 if k % 3 else 0.0}\n")
                f.write("2\n0 2.0 0.0 0.0 0.0 0.0\n5 1.5 0.5 1.0 -2.0 3.0\n")
    r = subprocess.run([FLUAM_REF, "data.main"], cwd=d, capture_output=True, text=True,
                       timeout=600)
    if "END" not in r.stdout:
        raise RuntimeError(f"{name}: reference run failed\n{r.stdout[-2000:]}")
    for ext in (".cuda", ".time", ".data.main"):
        os.remove(os.path.join(d, "out" + ext))
    if spec.get("fluid_only"):
        # the particle-free scheme writes its final field with the cells' full
        # 15 digits; keep the fixtures small
        assert os.path.getsize(os.path.join(d, "out.fluidFinalConfiguration")) < 400_000


if __name__ == "__main__":
    if not os.path.exists(FLUAM_REF):
        sys.exit("build oracle/_ref first (python oracle/ref_cpu/build_ref.py)")
    only = sys.argv[1:]  # case names; all cases when none are given
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        make_case(name, spec)
        print("golden", name)
