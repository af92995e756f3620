"""Host-side logic of libadfdtd.so against the oracle, and the C-ABI export
check.  No GPU: only host entry points are called."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "adfdtd.h")).read()
    return sorted(set(re.findall(r"^int\s+(adf_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol(adf):
    names = _declared_symbols()
    assert len(names) >= 20
    so = C.CDLL(adf.LIB_PATH)
    for n in names:
        assert hasattr(so, n), n
    # and the Python binding covers each of them
    from acoustic_disguising_b200 import _lib
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) <= bound


def _c_declarations():
    """{name: [parameter type]} of every entry point in include/adfdtd.h."""
    txt = open(os.path.join(ROOT, "include", "adfdtd.h")).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    out = {}
    for m in re.finditer(r"^int\s+(adf_\w+)\s*\(([^;]*?)\)\s*;", txt, flags=re.M | re.S):
        params = " ".join(m.group(2).split())
        types = []
        if params != "void":
            for p in params.split(","):
                p = p.strip()
                name = re.search(r"(\**)\s*(\w+)$", p)
                types.append((p[:name.start()] + name.group(1)).replace("const", "").replace(" ", ""))
        out[m.group(1)] = types
    return out


def test_ctypes_signatures_match_the_c_header(adf):
    """Every argument the binding declares has the C type include/adfdtd.h
    gives it: scalars by width and signedness, pointers as pointers, and a
    typed pointer to the same structure or scalar (c_void_p stands for any
    pointer)."""
    from acoustic_disguising_b200 import _lib as L

    scalars = {"int": C.c_int, "uint32_t": C.c_uint32, "int64_t": C.c_int64,
               "size_t": C.c_size_t, "double": C.c_double}
    structs = {"adf_domain": L.Domain, "adf_txgrid": L.TxGridC, "adf_cpml": L.CpmlC,
               "adf_gfmap": L.GfMapC, "adf_gf_request": L.GfRequestC,
               "adf_kh_desc": L.KhDescC}
    decl = _c_declarations()
    bound = {name: (res, args) for name, res, args in L.SIGNATURES}
    assert set(decl) == set(bound)
    for name, ctypes_ in decl.items():
        res, args = bound[name]
        assert res is C.c_int, name
        assert len(args) == len(ctypes_), name
        for i, (ct, a) in enumerate(zip(ctypes_, args)):
            where = f"{name} argument {i} ({ct})"
            if ct == "adf_step_cb":
                assert a is L.STEP_CB, where
            elif not ct.endswith("*"):
                assert a is scalars[ct], where
            elif a in (C.c_void_p, C.c_char_p):
                assert ct != "char*" or a is C.c_char_p, where
            else:
                assert hasattr(a, "_type_") and issubclass(a, C._Pointer), where
                base = ct[:-1]
                want = structs.get(base) or scalars.get(base) or (
                    C.c_void_p if base in ("adf_ctx*", "adf_server*") else None)
                assert a._type_ is want, where


def test_ctypes_structures_match_the_c_header(adf, tmp_path):
    """Every structure the binding passes through the C ABI has the size and
    field offsets that include/adfdtd.h gives it (gcc on the header), so a
    field added on one side only is caught without a GPU."""
    import ctypes
    import shutil
    import subprocess

    from acoustic_disguising_b200 import _lib as L

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc is not available")
    pairs = [(L.Domain, "adf_domain"), (L.TxGridC, "adf_txgrid"), (L.CpmlC, "adf_cpml"),
             (L.GfRequestC, "adf_gf_request"), (L.KhDescC, "adf_kh_desc"),
             (L.GfMapC, "adf_gfmap")]
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "adfdtd.h"', "int main(void) {"]
    want = []
    for cls, cname in pairs:
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {name}));')
            want.append(getattr(cls, name).offset)
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    include = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([gcc, "-I", include, "-o", str(exe), str(src)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got == want


def test_no_cpu_fallback_without_gpu(adf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(adf.AdfError):
        adf.Context(0)


DOMS = [
    dict(tmax=4.0e-4, xmax=0.3, nx=51, cf=0.5),
    dict(tmax=799.5 * 4.2081e-6, xmax=0.2375, nx=96, c0=343.0, r0=1.2, cf=0.5),
    dict(tmax=1999.5 * 4.2081e-6, xmax=0.6375, nx=256, c0=343.0, r0=1.2, cf=0.5),
    dict(tmax=3e-3, xmax=0.13, ymax=0.2, zmax=0.11, nx=27, ny=41, nz=23, c0=343.0, r0=1.2,
         cf=0.5),
]


@pytest.mark.parametrize("kw", DOMS)
def test_domain_and_coords_bitwise(adf, oracle, kw):
    d = adf.Domain(**kw)
    o = oracle.domain(**kw)
    for f, _ in d._fields_:
        assert getattr(d, f) == getattr(o, f), f
    for axis in range(3):
        for chan in range(4):
            assert np.array_equal(adf.coord(d, axis, chan), oracle.coords(o, axis, chan))
    assert np.array_equal(adf.t(d), oracle.time_axis(o))


@pytest.mark.parametrize("kw", DOMS)
def test_pack_transceivers_bitwise(adf, oracle, kw):
    d = adf.Domain(**kw)
    o = oracle.domain(**kw)
    rng = np.random.default_rng(5)
    ext = np.array([d.xmax, d.ymax, d.zmax])
    n = 37
    pts = rng.uniform(-0.97, 0.97, (n, 3)) * ext
    pts[0] = 0.0  # on-node point
    pts[1] = [d.xmax - 0.2 * d.dx, 0, 0]  # beyond the last interior node: out of bounds
    dirs = np.zeros((n, 4))
    dirs[:, 0] = rng.uniform(-1, 1, n)
    dirs[:, 1:] = rng.standard_normal((n, 3))
    tfs = rng.standard_normal((n, d.nt))
    txs = [adf.Transceiver(pts[i], dirs[i], tfs[i]) for i in range(n)]
    g = adf.transceivers_to_grid(d, txs)
    go = oracle.transceivers_to_grid(o, pts, dirs, tfs)
    for c in range(4):
        assert np.array_equal(g.idx[c], go.idx[c])
        assert np.array_equal(g.w[c], go.w[c])
        assert np.array_equal(g.src[c], go.src[c])
    assert np.array_equal(g.direction, go.dir)


def test_illumination_helpers(adf, oracle):
    for n, r in [(64, 30 * 0.005), (2048, 45 * 0.005), (4096, 0.25)]:
        p, nn = adf.fibonacci_sphere(n, r)
        po, no = oracle.fibonacci_sphere(n, r)
        assert np.allclose(p, po, rtol=0, atol=1e-15 * r)
        assert np.allclose(nn, no, rtol=0, atol=1e-15)
    kw = DOMS[1]
    d, o = adf.Domain(**kw), oracle.domain(**kw)
    tf, ts = adf.impulsive_wavelet(d, 2000.0)
    tfo, tso = oracle.impulsive_wavelet(o, 2000.0)
    assert ts == tso
    assert np.allclose(tf, tfo, rtol=1e-14, atol=1e-300)
    for inj in (False, True):
        assert np.allclose(adf.ricker_wavelet(d, 2000.0, inj), oracle.ricker_wavelet(o, 2000.0, inj),
                           rtol=1e-13, atol=1e-13)
