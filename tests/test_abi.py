"""C ABI and host-side logic, CPU only: the library builds, loads and exports
every symbol include/*.h declares, struct layouts match the
reference header, parameter validation mirrors the reference bindings, and
nothing computes without a GPU (no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
HEADERS = sorted(os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h"))


def _header_functions():
    names = set()
    for h in HEADERS:
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(fpe_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from fpe_option_b200 import _lib, build

    build.build_library()
    return _lib.load()


def test_exports_every_declared_symbol(lib):
    from fpe_option_b200 import _lib

    names = _header_functions()
    assert len(names) >= 26
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    assert sorted(_lib.EXPORTED) == names


def test_reference_struct_layouts():
    # reference cpp/include/fpe_engine.h:193-198
    from fpe_option_b200 import _lib

    assert C.sizeof(_lib.FpeVecResult) == 16
    assert C.sizeof(_lib.FpeVec2Result) == 32
    assert C.sizeof(_lib.FpeGridPtsResult) == 48
    assert C.sizeof(_lib.FpeMatResult) == 16
    assert C.sizeof(_lib.FpeGreeksResult) == 32
    assert C.sizeof(_lib.FpeOneshotResult) == 40


def test_header_compiles_as_c_and_cpp(tmp_path):
    import subprocess

    includes = "".join(f'#include "{os.path.basename(h)}"\n' for h in HEADERS)
    for comp, ext in (("gcc", "c"), ("g++", "cpp")):
        src = tmp_path / f"t.{ext}"
        src.write_text(includes + "int main(void){return 0;}\n")
        subprocess.run([comp, "-I", os.path.join(ROOT, "include"), "-c", str(src), "-o",
                        str(tmp_path / f"t_{ext}.o")], check=True)


def _has_gpu():
    import shutil
    import subprocess

    if not shutil.which("nvidia-smi"):
        return False
    return subprocess.run(["nvidia-smi", "-L"], capture_output=True).returncode == 0


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback(lib):
    import fpe_option_b200 as fpe

    assert lib.fpe_device_available() == 0
    assert not lib.fpe_compute_create(1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1, 8, 8, 0.0, 8,
                                      50, 0.0, 150.0)
    res = fpe._lib.FpeOneshotResult()
    k = (C.c_double * 1)(80.0)
    lib.fpe_price_oneshot(1.2, 0.05, 0.35, -0.4, 0.1, 0.6, 60.0, 0.1, k, 1, 0.0, 8, 8, 8, 50,
                          0.0, 150.0, C.byref(res))
    assert res.len == 0 and not res.price
    with pytest.raises(RuntimeError):
        fpe.price(K=80.0)
    with pytest.raises(RuntimeError):
        fpe.Compute(n_s=8, n_v=8)
    assert fpe.is_available() is False


def test_free_functions_accept_empty_results(lib):
    from fpe_option_b200 import _lib

    for cls, fn in ((_lib.FpeVecResult, lib.fpe_compute_free_vec),
                    (_lib.FpeVec2Result, lib.fpe_compute_free_vec2),
                    (_lib.FpeGridPtsResult, lib.fpe_compute_free_grid_pts),
                    (_lib.FpeMatResult, lib.fpe_compute_free_mat),
                    (_lib.FpeGreeksResult, lib.fpe_compute_free_greeks),
                    (_lib.FpeOneshotResult, lib.fpe_compute_free_oneshot)):
        r = cls()
        fn(C.byref(r))


@pytest.mark.parametrize("kw,msg", [
    (dict(n_s=1), "n_s"), (dict(n_v=300), "n_v"), (dict(kappa=-1.0), "Heston"),
    (dict(option_type=2, barrier=70.0), "barrier"), (dict(option_type=6, barrier=50.0), "barrier"),
    (dict(option_type=8, barrier=10.0), "barrier"), (dict(K=[]), "empty"), (dict(K=[-5.0]), "barrier"),
])
def test_parameter_validation_mirrors_reference(kw, msg):
    # src/bindings/_params.mojo:53-121 + option_types.mojo:13-32
    import fpe_option_b200 as fpe

    a = dict(kappa=1.2, theta=0.05, sigma=0.35, rho=-0.4, r=0.1, T=0.6, S0=60.0, V0=0.1, n_s=8,
             n_v=8, barrier=0.0, ot=8, s_min=0.0, s_max=180.0, K=[80.0])
    a.update({("ot" if k == "option_type" else k): v for k, v in kw.items()})
    with pytest.raises(ValueError, match=msg if msg != "barrier" else "option_type|barrier"):
        fpe._validate(a["kappa"], a["theta"], a["sigma"], a["rho"], a["r"], a["T"], a["S0"],
                      a["V0"], a["n_s"], a["n_v"], a["barrier"], a["ot"], a["s_min"], a["s_max"],
                      a["K"])


def test_option_type_names():
    import fpe_option_b200 as fpe

    assert fpe._option_type_int("down_and_out_call") == 2
    assert fpe._option_type_int(9) == 9
    with pytest.raises(ValueError):
        fpe._option_type_int("invalid")
    with pytest.raises(ValueError):
        fpe._option_type_int(10)
    with pytest.raises(ValueError):
        fpe.FpeParams(option_type="bogus")
    with pytest.raises(ValueError):
        fpe.FpeParams(n_s=1)
    with pytest.raises(ValueError):
        fpe._strikes([1.0] * 1025)


def test_dropin_import_alias():
    import fpe_engine

    assert hasattr(fpe_engine, "price") and hasattr(fpe_engine, "Compute")
    assert fpe_engine.Compute.__name__ == "Compute"


@pytest.mark.parametrize("cname", ["FpeContract", "FpeBatchOptions"])
def test_batch_struct_layouts_match_the_header(tmp_path, cname):
    """The ctypes mirrors of the batch structs have the C header's size and
    field offsets (a field added to one side only would shift the rest)."""
    import subprocess

    from fpe_option_b200 import _lib

    st = getattr(_lib, cname)
    fields = [f[0] for f in st._fields_]
    body = "".join(f'  printf("%zu\\n", offsetof({cname}, {f}));\n' for f in fields)
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "fpe_engine.h"\n'
                   f"int main(void) {{\n  printf(\"%zu\\n\", sizeof({cname}));\n{body}  return 0;\n}}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(st)
    assert out[1:] == [getattr(st, f).offset for f in fields]


def test_batch_options_map_every_field():
    """BatchOptions.to_c carries each Python field into the C struct (a field
    added to the struct but not mapped would silently stay zero)."""
    import dataclasses

    import fpe_option_b200 as fpe
    from fpe_option_b200 import _lib

    c_fields = {f[0] for f in _lib.FpeBatchOptions._fields_}
    py_fields = {f.name for f in dataclasses.fields(fpe.BatchOptions)}
    assert c_fields == py_fields
    vals = {}
    for i, f in enumerate(dataclasses.fields(fpe.BatchOptions)):
        if f.type in ("int", int):
            vals[f.name] = 3 + i
        elif f.type in ("bool", bool):
            vals[f.name] = True
        else:
            vals[f.name] = 0.25 + i
    o = fpe.BatchOptions(**vals).to_c()
    for name, v in vals.items():
        assert getattr(o, name) == (1 if v is True else v), name
