"""Loader of the golden fixtures in tests/golden/ (made by make_golden.py from
the reference's own stokesLimit sources built for the host)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def read_particles(path):
    """Parse a .particles / .velocityParticles file into {time: (3, np)}."""
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


def simple_cubic(np_, lx, ly, lz, dim=3):
    """src/simpleCubic.cpp:25-63 (dimension 3, or 2: one layer that the
    filling loop may still stack)."""
    if dim == 3:
        sigma = (lx * ly * lz / np_) ** (1.0 / 3.0)
        nz = int(lz / sigma) or 1
    else:
        sigma = (lx * ly / np_) ** 0.5
        nz = 1
    nx = int(lx / sigma) or 1
    ny = int(ly / sigma) or 1
    while nx * ny * nz < np_:
        if nx * ny * nz < np_:
            nx += 1
        if nx * ny * nz < np_:
            ny += 1
        if nx * ny * nz < np_:
            nz += 1
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    q = np.zeros((3, np_))
    n = 0
    for i in range(nz):
        for j in range(ny):
            for k in range(nx):
                if n < np_:
                    q[:, n] = ((k + 0.5) * dx - lx / 2.0, (j + 0.5) * dy - ly / 2.0,
                               (i + 0.5) * dz - lz / 2.0)
                    n += 1
    return q


def cases():
    """Cases with particles (an out.particles file)."""
    return sorted(d for d in os.listdir(GOLDEN)
                  if os.path.exists(os.path.join(GOLDEN, d, "out.particles")))


def fluid_cases():
    """Cases of the particle-free incompressible scheme."""
    return sorted(d for d in os.listdir(GOLDEN)
                  if os.path.exists(os.path.join(GOLDEN, d, "out.fluidFinalConfiguration"))
                  and not os.path.exists(os.path.join(GOLDEN, d, "out.particles")))


def read_fluid_final(path, nc):
    """The velocity [3][nc] of a .fluidFinalConfiguration file."""
    lines = open(path).read().split("\n")
    assert lines[11] == "Velocity"
    return np.array([lines[13 + 2 * i].split() for i in range(nc)], dtype=float).T.copy()


def load_fluid(name):
    from fluam_b200 import parse_data_main
    d = os.path.join(GOLDEN, name)
    cfg, run = parse_data_main(os.path.join(d, "data.main"))
    words = open(os.path.join(d, "data.main")).read().split()
    k = words.index("backgroundvelocity")
    v0 = [float(x) for x in words[k + 1:k + 4]]
    nc = cfg.mx * cfg.my * cfg.mz
    return dict(dir=d, cfg=cfg, run=run, v0=v0, nc=nc,
                v=read_fluid_final(os.path.join(d, "out.fluidFinalConfiguration"), nc),
                temperature=open(os.path.join(d, "out.temperature")).read(),
                seed=int(open(os.path.join(d, "out.seed")).read()))


def load(name):
    """Inputs and reference outputs of one golden case."""
    from fluam_b200 import parse_data_main
    d = os.path.join(GOLDEN, name)
    cfg, run = parse_data_main(os.path.join(d, "data.main"))
    words = open(os.path.join(d, "data.main")).read().split()
    if "coordinates" in words:
        with open(os.path.join(d, "start.coor")) as f:
            n = int(f.readline())
            q0 = np.array([f.readline().split() for _ in range(n)], dtype=float).T.copy()
    else:
        q0 = simple_cubic(run["numberparticles"], cfg.lx, cfg.ly, cfg.lz,
                          2 if cfg.scheme >= 2 else 3)
    bonds = None
    if "bondedForces" in words:
        with open(os.path.join(d, "bonds.dat")) as f:
            nb = int(f.readline())
            bb = np.array([f.readline().split() for _ in range(nb)], dtype=float).reshape(nb, 4)
            nf = int(f.readline())
            ff = np.array([f.readline().split() for _ in range(nf)], dtype=float).reshape(nf, 6)
        # bondedForcesVersion != 0: the old format, one line per bond end
        k = words.index("bondedForcesVersion") if "bondedForcesVersion" in words else -1
        directed = k >= 0 and int(words[k + 1]) != 0
        bonds = dict(bi=bb[:, 0].astype(np.int32), bj=bb[:, 1].astype(np.int32), k=bb[:, 2],
                     r0=bb[:, 3], fi=ff[:, 0].astype(np.int32), fk=ff[:, 1], fr0=ff[:, 2],
                     fxyz=ff[:, 3:6], directed=directed)
    _, pos = read_particles(os.path.join(d, "out.particles"))
    # the first-order scheme and quasi2D write no .velocityParticles
    # (src/saveParticles.cu:43-46); stokesLimit2D writes zeros there (its
    # particle velocity array is never set), which are not forces
    fv = os.path.join(d, "out.velocityParticles")
    frc = read_particles(fv)[1] if os.path.exists(fv) and cfg.scheme < 2 else None
    seed = int(open(os.path.join(d, "out.seed")).read())
    return dict(dir=d, cfg=cfg, run=run, q0=q0, bonds=bonds, pos=pos, frc=frc, seed=seed)


def sample_steps(run, scheme=0):
    """(step, steps taken) of each sample: after a step with step % samplefreq
    == 0 and step > 0 (src/runSchemeStokesLimit.cu:83, 280); for the
    quasi-2D family before each step with step >= 0 on the same condition,
    plus one after the last (src/runSchemeQuasi2D.cu:99-252)."""
    out = []
    step = -run["numstepsRelaxation"]
    taken = 0
    sf = run["samplefreq"]
    if scheme >= 2:
        while step < run["numsteps"]:
            if step >= 0 and step % sf == 0:
                out.append((step, taken))
            step += 1
            taken += 1
        if step % sf == 0:
            out.append((step, taken))
        return out
    while step < run["numsteps"]:
        step += 1
        taken += 1
        if step % sf == 0 and step > 0:
            out.append((step, taken))
    return out
