"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/pandora_gpu.h declares, agrees on the params layout, and rejects bad
parameters with the documented status codes before touching a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(pandora_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    import pandora
    L = pandora.load(build_if_missing=True)
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert _declared() <= set(pandora._lib.SIGNATURES), _declared() - set(pandora._lib.SIGNATURES)


def test_params_layout_and_defaults():
    import pandora
    L = pandora.load()
    assert L.pandora_params_sizeof() == ctypes.sizeof(pandora.Params)
    p = pandora.Params()
    assert L.pandora_params_default(ctypes.byref(p)) == 0
    q = pandora.default_params(32)
    for k, v in q.as_dict().items():
        assert getattr(p, k) == v, k


def test_sizes():
    import pandora
    L = pandora.load()
    p = pandora.default_params(64)
    a, b, c, k = (ctypes.c_int32() for _ in range(4))
    m = ctypes.c_int64()
    assert L.pandora_sizes(ctypes.byref(p), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                           ctypes.byref(m), ctypes.byref(k)) == 0
    assert (a.value, b.value, c.value, m.value) == (22, 43, 43, 22 * 43 * 43)
    assert k.value == round((3 * 21 ** 2) ** 0.5)


@pytest.mark.parametrize("field,value,status", [
    ("nodes_x", 100, -6),         # not 2^a x {1, 3, 5, 7} (2^2 * 5^2)
    ("rk3_cfl", 1.0, -7),         # g_RK3Check
    ("precision", 7, -10),
    ("f_type", 3, -10),           # RDT flow types are not in this library
    ("rk3_timestep", 9, -1),
])
def test_create_rejects_bad_params(field, value, status):
    import pandora
    L = pandora.load()
    p = pandora.default_params(32)
    setattr(p, field, value)
    h = ctypes.c_void_p()
    assert L.pandora_create(ctypes.byref(p), ctypes.byref(h)) == status
    assert not h.value


def test_create_without_device_fails_loudly():
    import pandora
    L = pandora.load()
    if pandora.device_count() > 0:
        pytest.skip("a device is present")
    p = pandora.default_params(32)
    h = ctypes.c_void_p()
    assert L.pandora_create(ctypes.byref(p), ctypes.byref(h)) == -9
    with pytest.raises(pandora.PandoraError):
        pandora.Simulation(p)


def test_strerror():
    import pandora
    L = pandora.load()
    for s in range(0, -11, -1):
        assert L.pandora_strerror(s)
