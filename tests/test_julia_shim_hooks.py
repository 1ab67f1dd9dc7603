"""The Julia binding names the library's hook implementations (no GPU, no
Julia): every implementation name the shim's gpu_hooks documentation and
INTEGRATION.md's example use is in the library's registry, and every
registry entry is documented in the shim, so a plugin author copying a name
from either gets a hook the library has."""
import ctypes as C
import os
import re

from frforge_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _registry():
    lib = L.load()
    out = set()
    for i in range(lib.frg_hook_count()):
        name, sl, hid, npar = C.c_char_p(), C.c_int(), C.c_int(), C.c_int()
        assert lib.frg_hook_info(i, C.byref(name), C.byref(sl), C.byref(hid), C.byref(npar)) == 0
        out.add(name.value.decode())
    return out


def test_shim_names_every_registry_entry():
    src = open(os.path.join(ROOT, "julia", "FRForgeCUDA.jl")).read()
    doc = src[src.index("gpu_hooks(method) ->"):src.index("gpu_hooks(::AbstractCapturingMethod)")]
    named = set(re.findall(r'"([a-z_]+)"', doc))
    assert named == _registry()


def test_integration_example_uses_registry_names():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    used = set(re.findall(r'gpu_hooks\([^)]*\) = \[\("([a-z_]+)"', text))
    used |= set(re.findall(r'"([a-z_]+)", sl, id\)', text))
    assert used and used <= _registry()
