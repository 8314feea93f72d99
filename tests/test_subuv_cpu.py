"""obit_dft_sub_uv argument checks that need no GPU: a call without fields, a
mode choice or gridded pass without the images are rejected with
OBIT_DFT_EBADARG and a message, before any device work; an unknown mode
never reaches the library."""
import numpy as np
import pytest

from obit_b200 import _lib
from obit_b200 import grid as GR
from obit_b200.comps import CCField, CCModel
from obit_b200.skymodel import SkyModelParams
from obit_b200.subuv import sub_uv
from obit_b200 import uvdata as U


def _uv():
    fa = U.freq_axis(8, 1, 1.4e9, 1e6)
    rng = np.random.default_rng(3)
    uvw = rng.uniform(-1e3, 1e3, (4, 3))
    return U.make_uvdata(uvw, 2, 8, 1, 1.4e9, fa, rng)


def _field():
    return CCField(flux=np.ones(3, np.float32), deltaX=np.zeros(3, np.float32), deltaY=np.zeros(3, np.float32),
                   crvalRA=0.0, crvalDec=30.0, do3D=False, cdeltX=-1e-4, cdeltY=1e-4)


def test_rejects_no_fields():
    with pytest.raises(_lib.DFTError) as e:
        sub_uv(_uv(), [], [], CCModel(uvRA=0.0, uvDec=30.0), SkyModelParams(), mode=GR.MODE_DFT)
    assert e.value.code == 1 and "no fields" in str(e.value)


def test_rejects_choice_and_grid_without_images():
    for mode in (GR.MODE_FASTEST, GR.MODE_GRID):
        with pytest.raises(_lib.DFTError) as e:
            sub_uv(_uv(), [_field()], [], CCModel(uvRA=0.0, uvDec=30.0), SkyModelParams(), mode=mode)
        assert e.value.code == 1 and "images" in str(e.value)


def test_rejects_unknown_mode():
    with pytest.raises(ValueError):
        sub_uv(_uv(), [_field()], [GR.GridImage(64, 64, 33, 33)], CCModel(uvRA=0.0, uvDec=30.0),
               SkyModelParams(), mode=7)
