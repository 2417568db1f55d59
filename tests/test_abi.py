"""The C-ABI library: symbols, data.main parsing, and failure without a GPU
(no compute calls here)."""
import ctypes
import os
import re

import pytest

from fluam_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(fsl_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) <= set(_lib.EXPORTS) | set(declared)
    missing = set(_lib.EXPORTS) - set(declared)
    assert not missing, missing


def test_config_layout_matches_header():
    # fsl_config: 4 int32, 9 doubles, 1 uint64, 10 int32, 5 doubles
    assert ctypes.sizeof(_lib.Config) == 4 * 4 + 9 * 8 + 8 + 10 * 4 + 5 * 8
    assert ctypes.sizeof(_lib.Status) == 8 + 4 + 4 + 8 + 4 + 4
    # fsl_class_tuning: 13 int32, 8 + 2 floats, 1 int32, 2 floats, 2 int32, 4 floats
    assert ctypes.sizeof(_lib.ClassTuning) == 13 * 4 + 10 * 4 + 4 + 2 * 4 + 2 * 4 + 4 * 4


def test_tuning_query_checks_arguments():
    L = _lib.load()
    t = _lib.ClassTuning()
    assert L.fsl_batch_get_class_tuning(None, 0, ctypes.byref(t)) == -1
    assert L.fsl_get_tuning(None, ctypes.byref(t)) == -1


def test_step_io_checks_arguments():
    """The input/output steps refuse a missing handle or buffer before they
    touch a device."""
    L = _lib.load()
    buf = (ctypes.c_double * 6)()
    assert L.fsl_step_io(None, buf, buf) == -1
    assert L.fsl_batch_step_io(None, buf, buf) == -1


def test_defaults_follow_reference():
    c = _lib.Config()
    _lib.load().fsl_config_defaults(ctypes.byref(c))
    assert c.kernel == 3 and c.pair == _lib.PAIR_TABLE_LJ and c.rfd == _lib.RFD_REFERENCE
    assert c.nonbonded == 1 and c.device == -1 and c.cutoff == 0.0


DATA_MAIN = """#Chose scheme
stokesLimit
particles		1
numberparticles		256
cutoff                  1.5
maxNumberPartInCellNonBonded    20
maxNumberPartInCell     	20
densfluid               1
shearviscosity          1.25
temperature             0.01
cells			32	24	16
celldimension		32	24	16
initfluid 1
backgroundvelocity 	 0  	0	    0
savedensity 0 these words are skipped
seed			17
numstepsRelaxation	3
numsteps                100
samplefreq              10
savefreq		0
dt			0.01
outputname		{out}
extraMobility 0.5
kernelPoints 4
pairPotential soft
softEpsilon 2.0
rfdMode paper
"""


def test_parse_data_main(tmp_path):
    from fluam_b200 import parse_data_main
    p = tmp_path / "data.main"
    p.write_text(DATA_MAIN.format(out=tmp_path / "run"))
    c, run = parse_data_main(p)
    assert (c.mx, c.my, c.mz) == (32, 24, 16)
    assert (c.lx, c.ly, c.lz) == (32.0, 24.0, 16.0)
    assert c.shearviscosity == 1.25 and c.temperature == 0.01 and c.dt == 0.01
    assert c.cutoff == 1.5 and c.seed == 17 and c.extra_mobility == 0.5
    assert c.kernel == 4 and c.pair == _lib.PAIR_SOFT and c.soft_epsilon == 2.0
    assert c.rfd == _lib.RFD_PAPER
    assert run == {"numsteps": 100, "samplefreq": 10, "numstepsRelaxation": 3,
                   "numberparticles": 256}


def test_parse_rejects_unknown_keyword(tmp_path):
    from fluam_b200 import parse_data_main
    p = tmp_path / "data.main"
    p.write_text("stokesLimit\ncells 8 8 8\nnotAKeyword 3\n")
    with pytest.raises(_lib.FslError) as e:
        parse_data_main(p)
    assert e.value.code == -6


def test_parse_missing_file(tmp_path):
    from fluam_b200 import parse_data_main
    with pytest.raises(_lib.FslError) as e:
        parse_data_main(tmp_path / "nope")
    assert e.value.code == -5


def test_create_fails_loudly_without_device():
    """With no usable GPU the library reports a CUDA error; there is no CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fluam_b200 import StokesLimit, make_config
    import numpy as np
    c = make_config((8, 8, 8), (8, 8, 8), kT=0.01, dt=0.01, cutoff=1.5)
    with pytest.raises(_lib.FslError) as e:
        StokesLimit(c, np.zeros((3, 4)))
    assert e.value.code in (-2, -3)


def test_create_validates_before_touching_the_device():
    from fluam_b200 import StokesLimit, make_config
    import numpy as np
    bad = [make_config((13, 8, 8), (8, 8, 8), dt=0.01, cutoff=1.5),   # 13 is not 2,3,5,7,11-smooth
           make_config((8, 8, 8), (8, 8, 8), dt=0.0, cutoff=1.5),
           make_config((8, 8, 8), (8, 8, 8), dt=0.01, cutoff=0.0),     # LJ pairs need rc > 0
           make_config((8, 8, 8), (8, 8, 8), dt=0.01, cutoff=1.5, kernel=5)]
    for c in bad:
        with pytest.raises(_lib.FslError) as e:
            StokesLimit(c, np.zeros((3, 4)))
        assert e.value.code == -1


def test_batch_and_server_fail_loudly_without_device():
    """The batched and serving entry points have no CPU path either."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fluam_b200 import Batch, Server, make_config
    import numpy as np
    c = make_config((8, 8, 8), (8, 8, 8), kT=0.01, dt=0.01, cutoff=1.5)
    with pytest.raises(_lib.FslError) as e:
        Batch([c, c], [np.zeros((3, 4)), np.zeros((3, 2))])
    assert e.value.code in (-2, -3)
    with pytest.raises(_lib.FslError) as e:
        Server(hbm_budget=1 << 30)
    assert e.value.code in (-2, -3)


def test_batch_validates_every_instance():
    from fluam_b200 import Batch, make_config
    import numpy as np
    good = make_config((8, 8, 8), (8, 8, 8), kT=0.01, dt=0.01, cutoff=1.5)
    bad = make_config((13, 8, 8), (8, 8, 8), kT=0.01, dt=0.01, cutoff=1.5)
    with pytest.raises(_lib.FslError) as e:
        Batch([good, bad], [np.zeros((3, 4)), np.zeros((3, 4))])
    assert e.value.code == -1 and "instance 1" in str(e.value)
