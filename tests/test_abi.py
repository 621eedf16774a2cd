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
    assert _abi.lib().vdi_abi_version() == 2


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


def _cfg_lines(drop=()):
    return "\n".join(l for l in open(os.path.join(HERE, "golden", "id_vis32.cfg")).read().splitlines()
                     if l.split("#")[0].strip() not in drop) + "\n"


@pytest.mark.parametrize("r,drop", [(4e-4, ()), (1e-3, ()), (5e-3, ()), (4e-4, ("x_sym",)), (2e-3, ("x_sym",))])
def test_nif_range_window_matches_fileinfo(r, drop):
    """nif_range's column window is fileinfo.cc:179-191 with the grid's 1/dx
    (the reference reads fileinfo::xsp there, which no constructor sets)."""
    import vdropimpact_b200 as V
    txt = _cfg_lines(drop) + f"nif_range {r}\ntracers 7\n"
    p = V.params_from_cfg(txt)
    o = vo.parse_cfg(txt)
    assert (p.nif_mode, p.nif_a, p.nif_b) == (2, o.nif_a, o.nif_b)
    assert 0 <= p.nif_a < p.nif_b <= p.m - 1
    assert p.ntrace == 7 == o.ntrace
    c = V.params_from_cfg(_cfg_lines(drop) + "nif_center\n")
    assert (c.nif_mode, c.ntrace) == (1, 0)


def test_nif_range_window_too_small_is_a_config_error():
    import vdropimpact_b200 as V
    with pytest.raises(V.VdiError) as e:
        V.params_from_cfg(_cfg_lines() + "nif_range 1e-9\n")
    assert e.value.status == 9
    with pytest.raises(vo.OracleError):
        vo.parse_cfg(_cfg_lines() + "nif_range 1e-9\n")


def test_bad_config_is_an_error_not_an_exit():
    import vdropimpact_b200 as V
    with pytest.raises(V.VdiError) as e:
        V.params_from_cfg("grid_points 16 8\nbogus_keyword 1\n")
    assert e.value.status == 9 and "bogus_keyword" in str(e.value)
    with pytest.raises(V.VdiError):
        V.params_from_cfg("grid_points 16 8\n")
