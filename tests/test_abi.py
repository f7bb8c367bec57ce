"""The C-ABI library loads on a machine without a GPU and exports every entry
point that include/chimera_gpu.h declares; argument validation needs no device."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "chimera_gpu.h")


def declared_symbols(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(chimera_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from chimera_b200 import build, gpu
    if not os.path.exists(gpu.LIB_PATH):
        build.build()
    return gpu.lib()


def test_header_declares_entry_points():
    syms = declared_symbols(HEADER)
    for s in ("chimera_create", "chimera_step", "chimera_set_state", "chimera_get_state",
              "chimera_diag", "chimera_destroy", "chimera_batch_create", "chimera_strerror"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols(HEADER) if not hasattr(lib, s)]
    assert not missing, missing


def test_strerror(lib):
    from chimera_b200.gpu import ERR
    assert lib.chimera_strerror(0) == b"ok"
    assert b"invalid" in lib.chimera_strerror(-1)
    assert lib.chimera_strerror(12345) == b"unknown error"
    texts = [lib.chimera_strerror(code) for code in ERR]     # every error code has its own text
    assert b"unknown error" not in texts and len(set(texts)) == len(ERR)


def _cfg(**kw):
    from chimera_b200 import gpu
    from chimera_b200.config import SolverConfig
    base = dict(nx=16, ny=16, dx=1 / 16, dy=1 / 16, gamma=5 / 3)
    base.update(kw)
    return gpu.to_ccfg(SolverConfig(**base))


@pytest.mark.parametrize("kw,code", [
    (dict(nx=3), -1),                  # N >= 4 (src/mhd_init.f90:208)
    (dict(dx=0.0), -1),
    (dict(gamma=1.0), -1),
    (dict(riemann=4), -1),
    (dict(limiter=0), -1),
    (dict(bc=(1, 1, 5, 5)), -1),
])
def test_create_rejects_bad_config(lib, kw, code):
    h = C.c_void_p()
    cfg = _cfg(**kw)
    assert lib.chimera_create(C.byref(cfg), None, C.byref(h)) == code
    assert not h.value


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("bc", [(1, 3, 1, 1), (3, 1, 2, 1), (1, 4, 3, 1)])
def test_create_accepts_mixed_pairs(lib, precision, bc):
    """A periodic side facing a non-periodic one passes the argument checks in
    every precision form (the reference takes each side on its own): creation
    succeeds on a GPU and stops at the device check without one."""
    h = C.c_void_p()
    cfg = _cfg(bc=bc, precision=precision)
    rc = lib.chimera_create(C.byref(cfg), None, C.byref(h))
    assert rc in (0, -6), rc
    if rc == 0:
        lib.chimera_destroy(h)


def test_null_arguments(lib):
    h = C.c_void_p()
    assert lib.chimera_create(None, None, C.byref(h)) == -1
    assert lib.chimera_step(None, 1) == -1
    assert lib.chimera_diag(None, None) == -1
    P = C.c_void_p
    # y-slab and dt hand-off entry points: a null handle is refused before any device call
    assert lib.chimera_halo_pack(None, C.c_int(7), P(0), P(0)) == -1
    assert lib.chimera_halo_unpack(None, C.c_int(7), P(0), P(0)) == -1
    assert lib.chimera_slab_ghost_rows(None, C.c_int(7), C.c_int(7)) == -1
    assert lib.chimera_refresh_dt(None, P(0)) == -1
    assert lib.chimera_get_dt_device(None, P(0)) == -1
    assert lib.chimera_set_dt_device(None, P(0)) == -1
    lib.chimera_destroy(None)


FORTRAN = os.path.join(ROOT, "chimera_b200", "fortran", "chimera_gpu_iface.f90")


def _c_arities(path):
    """name -> number of parameters of every prototype in the header."""
    text = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(chimera_\w+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        p = params.strip()
        out[name] = 0 if p in ("", "void") else p.count(",") + 1
    return out


def _fortran_arities(path):
    """bind(C) name -> number of dummy arguments in the interface module."""
    text = open(path).read().replace("&\n", " ")
    out = {}
    for args, name in re.findall(r"(?:function|subroutine)\s+\w+\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)",
                                 text):
        out[name] = len([a for a in args.split(",") if a.strip()])
    return out


def test_fortran_module_binds_every_entry_point_with_its_arity():
    c, f = _c_arities(HEADER), _fortran_arities(FORTRAN)
    assert set(c) == set(declared_symbols(HEADER))
    assert sorted(set(c) - set(f)) == []
    assert sorted(set(f) - set(c)) == []
    assert {k: f[k] for k in c if f[k] != c[k]} == {}


def test_host_arrays_pass_with_their_pitch():
    """A view of a padded float64 host array goes to the library as it is
    (pointer of the view, its row pitch as ld): an output written there lands
    in the caller's array, not in a copy."""
    import numpy as np
    from chimera_b200.gpu import HOST, _ptrs
    big = [np.zeros((9, 13)) for _ in range(6)]
    views = [b[:8, :10] for b in big]
    p, ld, where, _ = _ptrs(views, 10, 8, out=True)
    assert ld == 13 and where == HOST
    assert [x.value for x in p] == [v.ctypes.data for v in views]
    dense = [np.zeros((8, 10)) for _ in range(6)]
    assert _ptrs(dense, 10, 8, out=True)[1] == 10
    # inputs that are not float64 / not x-contiguous are converted; outputs are refused
    p, ld, _, keep = _ptrs([np.zeros((8, 10), dtype=np.float32)] * 6, 10, 8)
    assert ld == 10 and keep[0].dtype == np.float64
    with pytest.raises(ValueError):
        _ptrs([np.zeros((8, 10), dtype=np.float32)] * 6, 10, 8, out=True)
    with pytest.raises(ValueError):
        _ptrs([b[:8, :20:2] for b in [np.zeros((8, 20))] * 6], 10, 8, out=True)


@pytest.mark.parametrize("kw,code", [
    (dict(nx=1), -1),
    (dict(dy=0.0), -1),
    (dict(riemann=4), -1),
    (dict(bc=(1, 1, 5, 5)), -1),         # side values are 1..4 (src/mhd_config.f90:40-43)
    (dict(nx=50000, ny=50000), -8),      # (nx + 2)(ny + 2) beyond the kernels' int indices
])
def test_unit_ops_reject_bad_config(lib, kw, code):
    """The per-routine entry points check cfg before any device call (the
    pointers below are never dereferenced: each call returns first)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the refusal without a device")
    cfg = _cfg(**kw)
    P = C.c_void_p
    assert lib.chimera_op_average_face_to_cell_B(C.byref(cfg), P(8), P(8), P(8), P(8), None) == code
    assert lib.chimera_op_compute_divB(C.byref(cfg), P(8), P(8), P(8), None) == code


def test_misaligned_pointers_refused_before_any_device_call(lib):
    """Entry points whose kernels use the caller's arrays directly refuse a
    pointer that is not aligned for double (it would fault a launch).  With
    every pointer aligned the same calls get past the check and, on a machine
    without a GPU, stop at their first CUDA call instead."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the refusal without a device")
    cfg = _cfg()
    P = C.c_void_p
    good, odd = P(64), P(64 + 4)
    avg = lib.chimera_op_average_face_to_cell_B
    assert avg(C.byref(cfg), good, good, good, odd, None) == -1
    assert avg(C.byref(cfg), good, good, good, good, None) not in (0, -1)
    assert lib.chimera_op_compute_divB(C.byref(cfg), odd, good, good, None) == -1
    t, oc = C.c_double(0.0), C.c_int(1)
    step = lib.chimera_rk3_step_noalloc
    args = [good] * 6
    assert step(C.byref(cfg), *args, C.byref(t), C.byref(oc), None, None) not in (0, -1)
    args[2] = odd
    assert step(C.byref(cfg), *args, C.byref(t), C.byref(oc), None, None) == -1


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++11")])
def test_header_is_plain_c_and_cpp(lang, std, tmp_path):
    """include/chimera_gpu.h stands alone as C99 and C++11 (no CUDA headers), so
    C, C++ and Fortran-side build systems can use it as it is."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-x", lang, HEADER],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


_LAYOUT_C = r"""
#include <stddef.h>
#include <stdio.h>
#include "chimera_gpu.h"
#define F(S, f) printf(#S " " #f " %zu %zu\n", offsetof(S, f), sizeof(((S*)0)->f));
int main(void) {
  printf("chimera_cfg SIZE %zu 0\n", sizeof(chimera_cfg));
  printf("chimera_diag_out SIZE %zu 0\n", sizeof(chimera_diag_out));
  F(chimera_cfg, nx) F(chimera_cfg, ny) F(chimera_cfg, dx) F(chimera_cfg, dy) F(chimera_cfg, gamma)
  F(chimera_cfg, courant) F(chimera_cfg, t_out) F(chimera_cfg, t_end) F(chimera_cfg, bc_xlo)
  F(chimera_cfg, bc_xhi) F(chimera_cfg, bc_ylo) F(chimera_cfg, bc_yhi) F(chimera_cfg, riemann)
  F(chimera_cfg, limiter) F(chimera_cfg, use_slope_limiting) F(chimera_cfg, mood) F(chimera_cfg, precision)
  F(chimera_diag_out, t) F(chimera_diag_out, dt) F(chimera_diag_out, output_count)
  F(chimera_diag_out, active) F(chimera_diag_out, steps) F(chimera_diag_out, divb_max)
  F(chimera_diag_out, divb_mean) F(chimera_diag_out, bmax) F(chimera_diag_out, divb_rel)
  F(chimera_diag_out, mass) F(chimera_diag_out, energy) F(chimera_diag_out, cfl_speed)
  F(chimera_diag_out, mood_resets) F(chimera_diag_out, floor_hits) F(chimera_diag_out, status)
  return 0;
}
"""


def _c_layout(tmp_path):
    import shutil
    import subprocess
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / "layout.c"
    src.write_text(_LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        s, f, off, size = line.split()
        out.setdefault(s, []).append((f, int(off), int(size)))
    return out


def test_ctypes_structs_match_the_header(tmp_path):
    """The ctypes mirrors of chimera_cfg / chimera_diag_out (chimera_b200.gpu)
    have the header's field order, offsets, sizes and total size."""
    from chimera_b200 import gpu
    lay = _c_layout(tmp_path)
    for name, cls in (("chimera_cfg", gpu.CCfg), ("chimera_diag_out", gpu.CDiag)):
        size = [e for e in lay[name] if e[0] == "SIZE"][0][1]
        fields = [e for e in lay[name] if e[0] != "SIZE"]
        assert C.sizeof(cls) == size, name
        assert [f for f, _ in cls._fields_] == [f for f, _, _ in fields], name
        for f, off, sz in fields:
            assert getattr(cls, f).offset == off and getattr(cls, f).size == sz, (name, f)


def test_fortran_types_match_the_header(tmp_path):
    """The bind(C) derived types of the Fortran module list the header's fields
    in the same order with interoperable kinds of the same sizes."""
    lay = _c_layout(tmp_path)
    text = open(FORTRAN).read()
    kinds = {"c_int": 4, "c_double": 8, "c_long_long": 8}
    for name in ("chimera_cfg", "chimera_diag_out"):
        body = re.search(rf"type, bind\(C\) :: {name}\n(.*?)end type {name}", text, flags=re.S).group(1)
        got = []
        for line in body.splitlines():
            m = re.match(r"\s*(?:integer|real)\((c_\w+)\)\s*::\s*(.+)", line)
            if m:
                got += [(f.strip(), kinds[m.group(1)]) for f in m.group(2).split(",")]
        want = [(f, sz) for f, _, sz in lay[name] if f != "SIZE"]
        assert got == want, name


def _c_conventions(path):
    """name -> (return kind, [per-parameter 'ptr' | 'val']) of every prototype."""
    text = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
    text = re.sub(r"#.*", "", text)
    out = {}
    for ret, name, params in re.findall(r"([A-Za-z_][\w\s\*]*?)\b(chimera_\w+)\s*\(([^;{]*?)\)\s*;", text,
                                        flags=re.S):
        ret = ret.split(";")[-1].split("}")[-1].strip()
        rk = "sub" if ret == "void" else ("ptr" if "*" in ret else "int")
        p = params.strip()
        kinds = [] if p in ("", "void") else [("val", "ptr", "ptr2")[min(a.count("*"), 2)] for a in p.split(",")]
        out[name] = (rk, kinds)
    return out


def _fortran_conventions(path):
    """bind(C) name -> (return kind, [per-argument 'val' | 'ptr' | 'ptr2']):
    with the value attribute an argument is a scalar, or a pointer if it is a
    type(c_ptr); without it the argument's address is passed -- a pointer, or
    a pointer to a pointer for a type(c_ptr) (an array of them included)."""
    text = open(path).read().replace("&\n", " ")
    out = {}
    pat = re.compile(r"^\s*(integer\(c_int\)\s+function|type\(c_ptr\)\s+function|subroutine)\s+\w+\s*"
                     r"\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)(.*?)^\s*end\s+(?:function|subroutine)",
                     flags=re.S | re.M)
    for head, args, name, body in pat.findall(text):
        rk = "sub" if head.startswith("subroutine") else ("ptr" if head.startswith("type") else "int")
        decl = {}
        for m in re.finditer(r"^\s*(type\(\w+\)|integer\(\w+\)|real\(\w+\))([^:\n]*)::\s*(.+)$", body, flags=re.M):
            typ, attrs, names = m.groups()
            for nm in re.sub(r"\([^)]*\)", "", names).split(","):
                byval, cptr = "value" in attrs, typ == "type(c_ptr)"
                decl[nm.strip()] = ("ptr" if cptr else "val") if byval else ("ptr2" if cptr else "ptr")
        out[name] = (rk, [decl[a.strip()] for a in args.split(",") if a.strip()])
    return out


def test_fortran_module_passes_every_argument_as_the_header_takes_it():
    """Scalars by value where the C parameter is a scalar; one level of
    address (a type(c_ptr) by value, or another argument by reference) where it
    is a pointer; a type(c_ptr) by reference where it is a pointer to a
    pointer; and the header's return kinds (int / pointer / none)."""
    c, f = _c_conventions(HEADER), _fortran_conventions(FORTRAN)
    assert set(f) == set(c), sorted(set(c) ^ set(f))
    assert {k: (c[k], f[k]) for k in c if c[k] != f[k]} == {}


def _c_params(path):
    """name -> (return text, [(level of indirection, base type)]) of every prototype."""
    text = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
    text = re.sub(r"#.*", "", text)
    out = {}
    for ret, name, params in re.findall(r"([A-Za-z_][\w\s\*]*?)\b(chimera_\w+)\s*\(([^;{]*?)\)\s*;", text,
                                        flags=re.S):
        ret = ret.split(";")[-1].split("}")[-1].strip()
        p = params.strip()
        plist = []
        if p not in ("", "void"):
            for a in p.split(","):
                words = a.replace("*", " ").replace("const", " ").split()
                plist.append((a.count("*"), " ".join(words[:-1])))
        out[name] = (ret, plist)
    return out


def test_ctypes_argtypes_match_the_header(lib):
    """Every argtypes / restype the Python bindings declare (chimera_b200.gpu,
    .ops, .adjoint) agrees with the header: int and double scalars as c_int
    and c_double, pointers as pointers, pointers to pointers as arrays of or
    pointers to c_void_p (an opaque c_void_p is accepted for either)."""
    from chimera_b200 import adjoint, ops
    ops._lib()
    adjoint._lib()
    scalars = {"int": C.c_int, "double": C.c_double}
    checked = 0
    for name, (ret, params) in _c_params(HEADER).items():
        fn = getattr(lib, name)
        if fn.argtypes is None:
            continue
        checked += 1
        assert len(fn.argtypes) == len(params), name
        for k, (t, (level, base)) in enumerate(zip(fn.argtypes, params)):
            if level == 0:
                assert t is scalars[base], (name, k)
            elif t is C.c_void_p or t is C.c_char_p:
                continue
            elif level == 1:
                assert issubclass(t, C._Pointer) and t._type_ is not C.c_void_p, (name, k)
            else:
                ok_array = issubclass(t, C.Array) and t._type_ is C.c_void_p
                ok_ptr = issubclass(t, C._Pointer) and t._type_ is C.c_void_p
                assert ok_array or ok_ptr, (name, k)
        if ret == "void":
            assert fn.restype is None, name
        elif "*" in ret:
            assert fn.restype in (C.c_void_p, C.c_char_p), name
        else:
            assert fn.restype is C.c_int, name
    assert checked >= 40


def test_constants_agree_across_the_bindings():
    """The header's switch, location, precision and error constants have the
    same values in the Python package and the Fortran module."""
    from chimera_b200 import config, gpu
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    h = {k: int(v) for k, v in re.findall(r"#define\s+(CHIMERA_\w+)\s+(-?\d+)\s*$", text, flags=re.M)}
    py = {
        "CHIMERA_RIEMANN_RUSANOV": config.RUSANOV, "CHIMERA_RIEMANN_HLLE": config.HLLE,
        "CHIMERA_RIEMANN_HLLD": config.HLLD, "CHIMERA_LIMITER_VAN_LEER": config.VAN_LEER,
        "CHIMERA_LIMITER_MC": config.MC, "CHIMERA_BC_PERIODIC": config.BC_PERIODIC,
        "CHIMERA_BC_FIXED": config.BC_FIXED, "CHIMERA_BC_OUTFLOW": config.BC_OUTFLOW,
        "CHIMERA_BC_INFLOW": config.BC_INFLOW, "CHIMERA_FP64": config.FP64,
        "CHIMERA_FP32_BULK": config.FP32_BULK, "CHIMERA_FP32_MIXED": config.FP32_MIXED,
        "CHIMERA_HOST": gpu.HOST, "CHIMERA_DEVICE": gpu.DEVICE,
        "CHIMERA_OK": gpu.OK,
    }
    py.update({name: code for code, name in gpu.ERR.items()})
    assert {k: (h.get(k), v) for k, v in py.items() if h.get(k) != v} == {}
    assert sorted(k for k in h if k.startswith("CHIMERA_ERR_")) == sorted(gpu.ERR.values())
    f = {}
    for decl in re.findall(r"parameter\s*::\s*(.+)", open(FORTRAN).read()):
        for name, val in re.findall(r"(CHIMERA_\w+)\s*=\s*(-?\d+)", decl):
            f[name] = int(val)
    assert f and {k: (h.get(k), v) for k, v in f.items() if h.get(k) != v} == {}
