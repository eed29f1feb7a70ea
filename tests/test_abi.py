"""The C-ABI library without a GPU: it loads, exports every symbol that
include/cgx.h declares, reports errors as statuses, and its host-side
MatrixMarket I/O reproduces the reference reader (Matrix.cpp:13-111)."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import cgxx_b200 as cg
from cgxx_b200 import _lib
from cgxx_b200 import generators as G
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(REPO, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(cgx_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declared_symbols():
    assert declared_symbols() <= set(_lib.PROTOTYPES)


def test_version_and_status_strings():
    lib = cg.load()
    a, b = C.c_int(), C.c_int()
    lib.cgx_version(C.byref(a), C.byref(b))
    assert (a.value, b.value) == (1, 0)
    assert lib.cgx_status_string(0) == b"success"
    assert lib.cgx_status_string(2) == b"invalid state"


def test_default_options_match_reference_defaults():
    o = cg.default_options()
    assert o.max_iterations == 1000 and o.tolerance == 1e-9  # CG.h:67,70
    assert o.preconditioner == cg.PRECOND_JACOBI and o.precision == cg.PRECISION_FP64


def test_errors_are_statuses():
    lib = cg.load()
    assert lib.cgx_gnn_set_probes(None, 0, 0, 1.0, 0) == 1
    assert lib.cgx_learned_capture_residual(None, 0) == 1
    assert lib.cgx_inner_band(None, None, None) == 1
    assert lib.cgx_inner_matvec(None, None, None) == 1
    assert lib.cgx_learned_apply(None, None, None) == 1
    with pytest.raises(cg.CgxError) as e:
        _lib.check(lib.cgx_create(C.byref(C.c_void_p()), -1))
    assert e.value.status == 1
    assert "no CUDA device" in e.value.message
    # NULL handle
    assert lib.cgx_solve(None, None, None) == 1
    assert lib.cgx_destroy(None) == 0


@pytest.mark.skipif(cg.device_count() > 0, reason="machine has a GPU")
def test_no_device_is_reported_not_faked():
    assert cg.device_count() == 0
    with pytest.raises(cg.CgxError):
        cg.Handle(0)


@pytest.mark.parametrize("name", ["poisson16.mtx", "spd_ragged300.mtx", "diffusion27_8.mtx"])
def test_native_reader_matches_reference_reader(name):
    p = os.path.join(GOLD, name)
    N, I, J, V = cg.mtx_read(p)
    st, N2, I2, J2, V2 = O.read_mtx(p)
    assert st == 0 and N == N2
    assert np.array_equal(I, I2) and np.array_equal(J, J2) and np.array_equal(V, V2)


def test_native_reader_error_messages_match_reference():
    runs = json.load(open(os.path.join(GOLD, "reference_runs.json")))
    for e in runs["errors"]:
        if e["env"]:
            continue
        with pytest.raises(cg.CgxError) as ex:
            cg.mtx_read(os.path.join(GOLD, e["file"]))
        assert ex.value.message == e["stderr"]


def test_native_writer_round_trip(tmp_path):
    A = G.diffusion3d(9, stencil=27, seed=8)
    p1, p2 = str(tmp_path / "a.mtx"), str(tmp_path / "b.mtx")
    G.write_mtx_symmetric(p1, A)
    G.write_mtx_symmetric_py(p2, A)
    assert open(p1, "rb").read() == open(p2, "rb").read()
    N, I, J, V = cg.mtx_read(p1)
    I2, J2, V2 = G.symmetric_file_coo(A)
    assert np.array_equal(I, I2) and np.array_equal(J, J2) and np.array_equal(V, V2)


def test_reader_many_threads_large(tmp_path):
    # Big enough that the parallel reader splits the file across threads.
    A = G.diffusion3d(40, stencil=7, seed=2)
    p = str(tmp_path / "big.mtx")
    G.write_mtx_symmetric(p, A)
    N, I, J, V = cg.mtx_read(p)
    st, N2, I2, J2, V2 = O.read_mtx(p)
    assert np.array_equal(I, I2) and np.array_equal(J, J2) and np.array_equal(V, V2)


def test_reader_rejects_missing_diagonal(tmp_path):
    p = tmp_path / "nodiag.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 3\n1 1 1\n2 1 1\n3 3 1\n")
    with pytest.raises(cg.CgxError) as e:
        cg.mtx_read(str(p))
    assert e.value.status == 7
