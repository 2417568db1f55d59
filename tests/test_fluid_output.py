"""Fluid output files (opt-in extension of the Stokes path, which in the
reference writes none): the text format of saveFluidFinalConfiguration
(src/saveFluidFinalConfiguration.cu:30-75) and the legacy ASCII VTK layout of
the reference's VTK writer (src/saveFluidVTK.cu:33-250,
src/visit_writer.c:321-460, 899-1015), restated here independently and
compared byte for byte with the library's writers.  No GPU needed.
"""
import ctypes

import numpy as np
import pytest

from fluam_b200 import _lib


def _vtk_expected(mx, my, mz, v):
    """The layout: header, DIMENSIONS, three coordinate sections, CELL_DATA
    with the cell-centred velocity; numbers as '%20.12e ' with a break after
    every ninth of a run."""
    out, col = [], [0]

    def num(x):
        out.append("%20.12e " % x)
        col[0] += 1
        if col[0] % 9 == 0:
            out.append("\n")
            col[0] = 0

    def section():
        if col[0]:
            out.append("\n")
            col[0] = 0

    out.append("# vtk DataFile Version 2.0\nWritten using VisIt writer\nASCII\n")
    out.append("DATASET RECTILINEAR_GRID\n")
    dims = (mx + 1, my + 1, mz + 1)
    out.append("DIMENSIONS %d %d %d\n" % dims)
    for a, name in enumerate("XYZ"):
        if a:
            section()
        out.append("%s_COORDINATES %d double\n" % (name, dims[a]))
        for i in range(dims[a]):
            num(float(i))
    section()
    nc = mx * my * mz
    out.append("CELL_DATA %d\nVECTORS velocity double\n" % nc)
    vx, vy, vz = (v[c].reshape(mz, my, mx) for c in range(3))
    cx = 0.5 * (np.roll(vx, 1, axis=2) + vx)
    cy = 0.5 * (np.roll(vy, 1, axis=1) + vy)
    cz = 0.5 * (np.roll(vz, 1, axis=0) + vz)
    for a, b, c in zip(cx.ravel(), cy.ravel(), cz.ravel()):
        num(a)
        num(b)
        num(c)
    out.append("\n")
    out.append("\n")
    return "".join(out)


@pytest.mark.parametrize("m", [(3, 4, 5), (6, 3, 4)])
def test_vtk_layout(tmp_path, m):
    mx, my, mz = m
    v = np.random.default_rng(1).standard_normal((3, mz * my * mx))
    path = tmp_path / "f.vtk"
    L = _lib.load()
    rc = L.fsl_write_fluid_vtk(str(path).encode(), mx, my, mz, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0
    assert path.read_text() == _vtk_expected(mx, my, mz, v)


def _cxx_g15(x):
    """std::ostream with precision(15), default float field: %.15g"""
    return "%.15g" % x


def test_fluid_final_configuration_format(tmp_path):
    L = _lib.load()
    c = _lib.Config()
    L.fsl_config_defaults(ctypes.byref(c))
    c.mx, c.my, c.mz = 3, 2, 2
    c.lx, c.ly, c.lz = 3.0, 2.5, 2.0
    c.temperature = 0.01
    v = np.random.default_rng(2).standard_normal((3, 12))
    p = np.array([1.0, 0.5, 0.25])
    path = tmp_path / "out.fluidFinalConfiguration"
    rc = L.fsl_write_fluid_final(str(path).encode(), ctypes.byref(c), 1.0,
                                 p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0,
                                 v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0
    lines = path.read_text().split("\n")
    assert lines[:12] == ["Number of cells 12", "mx my mz", "3 2 2", "lx ly lz", "3 2.5 2", "Density 1",
                          "Pressure parameters 1 0.5 0.25", "Thermostat 0", "Temperature 0.01",
                          "Cells properties ", "Density ", "Velocity"]
    body = lines[12:-1]
    assert len(body) == 24
    for i in range(12):
        assert body[2 * i] == "1"
        assert body[2 * i + 1] == " ".join(_cxx_g15(v[k, i]) for k in range(3))


def test_data_main_fluid_keywords_parse(tmp_path):
    (tmp_path / "data.main").write_text(
        "stokesLimit\nparticles 1\ncells 8 8 8\ncelldimension 8 8 8\nnumberparticles 8\n"
        "dt 0.01\nnumsteps 4\nsamplefreq 2\nsavefreq 2\nsaveFluid 1\nsaveVTK 1\n"
        "densfluid 1\npressureparameters 1 0 0\noutputname out\n")
    import fluam_b200
    c, run = fluam_b200.parse_data_main(tmp_path / "data.main")
    assert c.mx == 8 and run["samplefreq"] == 2
