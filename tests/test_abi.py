"""The C-ABI library loads, exports every entry point include/aturan_b200.h declares, agrees with
the Python mirror of its parameter struct, and fails loudly (no CPU fallback) without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

from aturan_b200 import api, params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aturan_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|const char\*)\s+(aturan_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = api.load_library()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
        assert n in api.SIGNATURES, n


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "aturan_b200.h"\n'
                   'int main(void){ printf("%zu %zu %zu %zu\\n", sizeof(aturan_params), offsetof(aturan_params, r0),'
                   ' offsetof(aturan_params, gas), sizeof(aturan_gas)); return 0; }\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, off_r0, off_gas, gsize = map(int, subprocess.check_output([str(exe)]).split())
    assert size == ctypes.sizeof(P.Params)
    assert off_r0 == P.Params.r0.offset
    assert off_gas == P.Params.gas.offset
    assert gsize == ctypes.sizeof(P.Gas)


def test_library_defaults_equal_python_defaults():
    a, b = api.library_default_params(), P.default_params()
    assert bytes(a) == bytes(b)


def test_post_params_layout_and_defaults(tmp_path):
    """aturan_post_params: the header's layout, and the library's defaults (the reference's knobs
    with the environment unset) equal the Python mirror's."""
    src = tmp_path / "pp.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "aturan_b200.h"\n'
                   'int main(void){ printf("%zu %zu %zu\\n", sizeof(aturan_post_params),'
                   ' offsetof(aturan_post_params, damp_t_horiz), offsetof(aturan_post_params, vel_shapiro));'
                   ' return 0; }\n')
    exe = tmp_path / "pp"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, off_h, off_v = map(int, subprocess.check_output([str(exe)]).split())
    assert size == ctypes.sizeof(P.PostParams)
    assert off_h == P.PostParams.damp_t_horiz.offset and off_v == P.PostParams.vel_shapiro.offset
    assert bytes(api.library_default_post_params()) == bytes(P.default_post_params())


def test_chem_params_layout_and_defaults(tmp_path):
    """aturan_chem_params: the header's layout, and the library's defaults (the reference's
    constants and knobs) equal the Python mirror's."""
    src = tmp_path / "cp.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "aturan_b200.h"\n'
                   'int main(void){ printf("%zu %zu %zu\\n", sizeof(aturan_chem_params),'
                   ' offsetof(aturan_chem_params, m_nh3), offsetof(aturan_chem_params, polar_floor));'
                   ' return 0; }\n')
    exe = tmp_path / "cp"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, off_m, off_f = map(int, subprocess.check_output([str(exe)]).split())
    assert size == ctypes.sizeof(P.ChemParams)
    assert off_m == P.ChemParams.m_nh3.offset and off_f == P.ChemParams.polar_floor.offset
    assert bytes(api.library_default_chem_params()) == bytes(P.default_chem_params())


def test_turb_params_layout_and_defaults(tmp_path):
    """aturan_turb_params: the header's layout, and the library's defaults equal the Python mirror's."""
    src = tmp_path / "tp.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "aturan_b200.h"\n'
                   'int main(void){ printf("%zu %zu %zu\\n", sizeof(aturan_turb_params),'
                   ' offsetof(aturan_turb_params, nue_max), offsetof(aturan_turb_params, nue_air));'
                   ' return 0; }\n')
    exe = tmp_path / "tp"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, off_m, off_a = map(int, subprocess.check_output([str(exe)]).split())
    assert size == ctypes.sizeof(P.TurbParams)
    assert off_m == P.TurbParams.nue_max.offset and off_a == P.TurbParams.nue_air.offset
    assert bytes(api.library_default_turb_params()) == bytes(P.default_turb_params())


def test_precip_params_layout_and_defaults(tmp_path):
    """aturan_precip_params: the header's layout, and the library's defaults equal the Python mirror's."""
    src = tmp_path / "pr.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "aturan_b200.h"\n'
                   'int main(void){ printf("%zu %zu\\n", sizeof(aturan_precip_params),'
                   ' offsetof(aturan_precip_params, rate_scale)); return 0; }\n')
    exe = tmp_path / "pr"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, off_r = map(int, subprocess.check_output([str(exe)]).split())
    assert size == ctypes.sizeof(P.PrecipParams) and off_r == P.PrecipParams.rate_scale.offset
    assert bytes(api.library_default_precip_params()) == bytes(P.default_precip_params())


def test_iter_params_layout_and_defaults(tmp_path):
    """aturan_iter_params: the header's layout (nested structs included), and the library's defaults
    equal the Python mirror's."""
    src = tmp_path / "ip.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "aturan_b200.h"\n'
                   'int main(void){ printf("%zu %zu %zu %zu\\n", sizeof(aturan_iter_params),'
                   ' offsetof(aturan_iter_params, omega), offsetof(aturan_iter_params, chem),'
                   ' offsetof(aturan_iter_params, precip)); return 0; }\n')
    exe = tmp_path / "ip"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    size, off_o, off_c, off_p = map(int, subprocess.check_output([str(exe)]).split())
    assert size == ctypes.sizeof(P.IterParams)
    assert (off_o, off_c, off_p) == (P.IterParams.omega.offset, P.IterParams.chem.offset, P.IterParams.precip.offset)
    assert bytes(api.library_default_iter_params()) == bytes(P.default_iter_params())


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.AturanError) as e:
        api.Context(P.default_params(im=9, jm=13, km=17))
    assert e.value.code == api.E_CUDA


def test_invalid_parameters_rejected():
    L = api.load_library()
    p = P.default_params()
    p.abi_version = 99
    h = ctypes.c_void_p()
    assert L.aturan_ctx_create(ctypes.byref(p), ctypes.byref(h)) == api.E_INVALID
    p = P.default_params(km=18)              # km-1 odd: colours would not alternate across the seam
    assert L.aturan_ctx_create(ctypes.byref(p), ctypes.byref(h)) == api.E_UNSUPPORTED
    assert L.aturan_ctx_create(None, ctypes.byref(h)) == api.E_INVALID
    pp = P.default_post_params()
    assert L.aturan_post_step(None, ctypes.byref(pp), None, None) == api.E_INVALID
    assert L.aturan_post_params_default(None) == api.E_INVALID
