"""The C-ABI library without a GPU: symbols, struct layout, defaults."""
import ctypes
import os
import re
import subprocess

import pytest

from simp_b200 import _lib, build
from simp_b200.params import SimpParams, reference_default

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("simp_gpu.h", "simp_serve.h")]


def declared_symbols():
    txt = "".join(open(h).read() for h in HEADERS)
    return sorted(set(re.findall(r"SIMP_API\s+[\w\s\*]*?\b(simp_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_params_layout_matches_c(tmp_path):
    fields = [f for f, _ in SimpParams._fields_]
    src = tmp_path / "layout.c"
    body = "\n".join(f'    printf("%s %zu\\n", "{f}", offsetof(simp_params, {f}));' for f in fields)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "simp_gpu.h"\nint main(void){\n'
                   f'    printf("sizeof %zu\\n", sizeof(simp_params));\n{body}\n    return 0;\n}}\n')
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    assert int(out["sizeof"]) == ctypes.sizeof(SimpParams)
    for f in fields:
        assert int(out[f]) == getattr(SimpParams, f).offset, f


@pytest.mark.parametrize("cname,pyname,header", [
    ("simp_forcing", "SimpForcing", "simp_gpu.h"),
    ("simp_server_config", "ServerConfig", "simp_serve.h"),
    ("simp_request_stats", "RequestStats", "simp_serve.h"),
    ("simp_server_stats", "ServerStats", "simp_serve.h"),
])
def test_struct_layouts_match_c(tmp_path, cname, pyname, header):
    from simp_b200 import params as P
    cls = getattr(P, pyname)
    fields = [f for f, _ in cls._fields_]
    src = tmp_path / "layout.c"
    body = "\n".join(f'    printf("%s %zu\\n", "{f}", offsetof({cname}, {f}));' for f in fields)
    src.write_text(f'#include <stddef.h>\n#include <stdio.h>\n#include "{header}"\nint main(void){{\n'
                   f'    printf("sizeof %zu\\n", sizeof({cname}));\n{body}\n    return 0;\n}}\n')
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    assert int(out["sizeof"]) == ctypes.sizeof(cls)
    for f in fields:
        assert int(out[f]) == getattr(cls, f).offset, f


def test_fortran_forcing_mirror_field_order():
    from simp_b200.params import SimpForcing
    src = open(os.path.join(ROOT, "fortran", "shim", "simp_gpu_mod.f90")).read()
    body = src[src.index("type, bind(C) :: simp_forcing"):src.index("end type simp_forcing")]
    names = []
    for line in body.splitlines()[1:]:
        if "::" in line:
            names += [n.strip() for n in line.split("::", 1)[1].split(",") if n.strip()]
    assert [n.lower() for n in names] == [f.lower() for f, _ in SimpForcing._fields_]


def test_fortran_interfaces_name_exported_symbols(lib):
    """Every bind(C, name=...) of the Fortran module is exported by the library."""
    src = open(os.path.join(ROOT, "fortran", "shim", "simp_gpu_mod.f90")).read()
    names = re.findall(r'bind\(C,\s*name="(simp_\w+)"\)', src)
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_fortran_shims_call_only_bound_entry_points():
    """The drop-in shims (time_integration, single_step) call only entry
    points the Fortran module binds."""
    mod = open(os.path.join(ROOT, "fortran", "shim", "simp_gpu_mod.f90")).read()
    bound = set(re.findall(r"(?:function|subroutine)\s+(simp_\w+)", mod))
    bound.add("simp_params_from_host")   # simp_host_params.f90
    for shim in ("time_integration_gpu.f90", "single_step_gpu.f90", "simp_host_params.f90"):
        src = open(os.path.join(ROOT, "fortran", "shim", shim)).read()
        code = "\n".join(line.split("!", 1)[0] for line in src.splitlines())
        used = set(re.findall(r"\b(simp_(?:gpu|params)_\w+)\s*\(", code))
        assert used, shim
        assert used <= bound, (shim, used - bound)


# simp_params members the reference has no variable for: the hard-coded
# wind and current (wind_forcing.f90:36-37, water_drag.f90:36-37) and the
# GPU's own settings
_NOT_FROM_HOST = {"wind_u", "wind_v", "current_u", "current_v", "vortex_x", "vortex_y", "vortex_umax",
                  "vortex_radius", "wind_kind", "precision", "skin", "mass_from_area", "reserved0",
                  "reserved1"}


def test_fortran_shims_take_the_hosts_parameters():
    """The drop-in shims build their simp_params from the host's modules:
    every member with a counterpart in globals.f90 / data_variables.f90 is
    assigned from the variable of the same name, and both shims use that
    routine rather than the library's compiled-in defaults."""
    src = open(os.path.join(ROOT, "fortran", "shim", "simp_host_params.f90")).read()
    code = "\n".join(line.split("!", 1)[0] for line in src.splitlines())
    assigned = {}
    for m in re.finditer(r"prm%(\w+)\s*=\s*(.+)", code):
        assigned[m.group(1).lower()] = m.group(2)
    for f, _ in SimpParams._fields_:
        if f in _NOT_FROM_HOST:
            continue
        assert f.lower() in assigned, f"simp_params%{f} is not taken from the host"
        assert re.search(rf"\b{f}\b", assigned[f.lower()], re.I), (f, assigned[f.lower()])
    for shim in ("time_integration_gpu.f90", "single_step_gpu.f90"):
        body = open(os.path.join(ROOT, "fortran", "shim", shim)).read()
        body = "\n".join(line.split("!", 1)[0] for line in body.splitlines())
        assert "call simp_params_from_host(prm)" in body, shim
        assert "simp_params_reference_default" not in body, shim


def test_fortran_mirror_field_order():
    """The bind(C) type in the Fortran shim lists the members in C order."""
    src = open(os.path.join(ROOT, "fortran", "shim", "simp_gpu_mod.f90")).read()
    body = src[src.index("type, bind(C) :: simp_params"):src.index("end type simp_params")]
    body = re.sub(r"&\s*\n\s*", " ", body)
    names = []
    for line in body.splitlines()[1:]:
        if "::" in line:
            names += [n.strip() for n in line.split("::", 1)[1].split(",") if n.strip()]
    assert [n.lower() for n in names] == [f.lower() for f, _ in SimpParams._fields_]


def test_reference_default_matches_python_mirror(lib):
    c = SimpParams()
    lib.simp_params_reference_default(ctypes.byref(c))
    py = reference_default()
    for f, _ in SimpParams._fields_:
        assert getattr(c, f) == getattr(py, f), f


def test_version_string(lib):
    assert b"sm_100a" in lib.simp_gpu_version()


def test_noalloc_rejects_bad_sizes_before_touching_the_device(lib):
    # n out of range and bad kernel codes are refused on the host
    assert lib.simp_gpu_sum_density_noalloc(1, 1, 1, 1, 0, 9, 1, None) == 1
    assert lib.simp_gpu_sum_density_noalloc(1, 1, 1, 1, 65537, 9, 1, None) == 1
    assert lib.simp_gpu_sum_density_noalloc(1, 1, 1, 1, 10, 10, 1, None) == 1


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(_lib.NativeLibraryMissing):
        _lib.load(str(tmp_path / "nope.so"))


def test_null_context_calls_are_refused(lib):
    assert lib.simp_gpu_step(None, 1, None, None) == 1
    assert lib.simp_gpu_destroy(None) == 0
    assert lib.simp_gpu_last_error(None) == b"null context"
