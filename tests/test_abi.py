"""CPU checks of the C ABI: the library loads, exports every entry point
include/vdi.h declares, and parses configuration text like fileinfo.cc."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import vdi_oracle as vo

HERE = os.path.dirname(os.path.abspath(__file__))


def test_library_exports_every_declared_symbol():
    from vdropimpact_b200 import _abi
    L = C.CDLL(_abi.LIB_PATH)
    declared = _abi.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    _abi.lib()  # binds every signature
    assert _abi.lib().vdi_abi_version() == 1


@pytest.mark.parametrize("cfg", ["id_vis32.cfg", "ld_vis100.cfg"])
def test_params_match_fileinfo(cfg):
    import vdropimpact_b200 as V
    text = open(os.path.join(HERE, "golden", cfg)).read()
    p = V.params_from_cfg(text)
    o = vo.parse_cfg(text)
    for a, b in (("m", "m"), ("n", "n"), ("ax", "ax"), ("bx", "bx"), ("by", "by"), ("mu", "mu"),
                 ("rho", "rho"), ("t_end", "t_end"), ("h0", "h0"), ("alpha", "alpha"), ("mug", "mug"),
                 ("Pamb", "Pamb"), ("R", "R"), ("V", "V"), ("sigma", "sigma"), ("tmult", "tmult")):
        assert getattr(p, a) == getattr(o, b), a
    assert p.x_sym == 1 and p.implicit_visc == 1 and p.nframes == 250


def test_bad_config_is_an_error_not_an_exit():
    import vdropimpact_b200 as V
    with pytest.raises(V.VdiError) as e:
        V.params_from_cfg("grid_points 16 8\nbogus_keyword 1\n")
    assert e.value.status == 9 and "bogus_keyword" in str(e.value)
    with pytest.raises(V.VdiError):
        V.params_from_cfg("grid_points 16 8\n")
