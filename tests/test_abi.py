"""The C-ABI shared library: it loads, exports every entry point that
include/wds_b200.h declares, and its struct layouts agree with the ctypes
mirror (checked by compiling the header with gcc).  No GPU needed."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wds_b200.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(wds_\w+)\s*\(", txt, re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    from wdsgpu_b200 import _lib
    lib = _lib.load()
    names = _declared()
    assert names, "no declarations parsed from the header"
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTS)


def test_struct_layout_matches_header(tmp_path):
    from wdsgpu_b200 import _lib
    src = tmp_path / "layout.c"
    fields = [f for f, _ in _lib.WdsNetwork._fields_]
    ofields = [f for f, _ in _lib.WdsForwardOpts._fields_]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wds_b200.h"',
             'int main(void){',
             'printf("%zu\\n", sizeof(WdsNetwork));',
             'printf("%zu\\n", sizeof(WdsForwardOpts));',
             'printf("%zu\\n", sizeof(WdsForwardIO));',
             'printf("%zu\\n", sizeof(WdsAdjointIO));']
    lines += ['printf("%%zu\\n", offsetof(WdsNetwork, %s));' % f for f in fields]
    lines += ['printf("%%zu\\n", offsetof(WdsForwardOpts, %s));' % f for f in ofields]
    lines += ['return 0;}']
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                           check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(_lib.WdsNetwork)
    assert vals[1] == ctypes.sizeof(_lib.WdsForwardOpts)
    assert vals[2] == ctypes.sizeof(_lib.WdsForwardIO)
    assert vals[3] == ctypes.sizeof(_lib.WdsAdjointIO)
    vals = vals[:2] + vals[4:]
    offs = vals[2:2 + len(fields)]
    for f, o in zip(fields, offs):
        assert getattr(_lib.WdsNetwork, f).offset == o, f
    for f, o in zip(ofields, vals[2 + len(fields):]):
        assert getattr(_lib.WdsForwardOpts, f).offset == o, f


def test_plan_without_a_device_fails_cleanly():
    """On a machine without a GPU, wds_plan returns an error code (never a
    crash) and the solver refuses CPU tensors instead of falling back."""
    import torch
    from wdsgpu_b200 import synth
    from wdsgpu_b200.solver import GGASolver
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = GGASolver(synth.config1_network(), device="cpu")
    with pytest.raises(NotImplementedError):
        s.solve(s.net.demand_cfs_at(0), s.net.reservoir_head_ft_at(0))
