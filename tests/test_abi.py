"""The C-ABI library loads and exports every entry point include/lima_b200.h
declares; host-side argument checks work without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lima_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^LIMA_API\s+[\w\s\*]+?\b(lima_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "lima_create" in names and "lima_step" in names and len(names) >= 30


def test_library_exports_every_declared_symbol():
    from lima_b200 import engine
    lib_path = engine.LIB_PATH
    assert os.path.exists(lib_path), "build liblima_b200.so first (python -m lima_b200.build)"
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (lima_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    # the binding covers the same set
    assert sorted(engine.EXPORTED) == declared_functions()
    lib = ctypes.CDLL(lib_path)
    for n in declared_functions():
        getattr(lib, n)


def test_default_params_and_errors_without_device():
    from lima_b200 import engine as E
    lib = E.load_library()
    p = E.default_params()
    assert p.nstlist == 10 and abs(p.dt - 1e-6) < 1e-18 and p.electrostatics == E.ES_EWALD
    # automatic pruning and pair-kernel row split, eager launches by default
    assert p.prune_interval < 0 and p.pair_split < 0 and p.use_graphs == 0
    assert lib.lima_error_string(E.LIMA_OK) == b"ok"
    h = ctypes.c_void_p()
    assert lib.lima_create(ctypes.byref(p), ctypes.byref(h)) == 0
    # argument checks happen on the host
    assert lib.lima_set_box(h, -1.0, 1.0, 1.0) == 1
    assert lib.lima_select_system(h, 3) == 1
    assert lib.lima_step(h, -1) == 1
    assert lib.lima_set_electric_field(h, float("nan"), 0.0, 0.0) == 1
    assert lib.lima_set_electric_field(h, 0.5, 0.0, 0.0) == 0
    bad = E.default_params(dt=0.0)
    h2 = ctypes.c_void_p()
    assert lib.lima_create(ctypes.byref(bad), ctypes.byref(h2)) == 1
    assert lib.lima_destroy(h) == 0


def test_no_silent_fallback_without_gpu():
    """Without a device the engine fails loudly instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lima_b200 import Engine, LimaError, systems
    s = systems.config0()
    e = Engine(cutoff=1.2, electrostatics=1)
    e.load(s)
    with pytest.raises(LimaError) as ex:
        e.compute_forces()
    assert ex.value.code == 6


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of lima_params, lima_energies and lima_timings have the
    header's sizes and field offsets (a C program compiled against the header
    prints them)."""
    from lima_b200 import engine as E
    structs = {"lima_params": E.Params, "lima_energies": E.Energies, "lima_timings": E.Timings,
               "lima_pairlist_stats": E.PairlistStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lima_b200.h"', 'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['    return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
