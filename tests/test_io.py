"""Parallel loaders of the reference's text files (csrc/sr_io.cpp) against the
reference's own readers compiled unchanged (load_data_file and
parse_input_info, src/utils/utils.cpp:122-300, through oracle/_ref) and the
plain Python readers: identical numbers, bit for bit."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle
from symbolic_regression_gpu_b200 import SrError, formats, synth

needs_ref = pytest.mark.skipif(not oracle.reference_available(),
                               reason="reference oracle not built")


def _ref():
    lib = oracle._ref_lib()
    lib.ref_load_data.restype = None
    lib.ref_load_data.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double)]
    P = ctypes.POINTER
    lib.ref_parse_gen.restype = ctypes.c_int
    lib.ref_parse_gen.argtypes = [ctypes.c_char_p, P(ctypes.c_int), P(ctypes.c_longlong),
                                  P(ctypes.c_int), P(ctypes.c_double), P(ctypes.c_longlong),
                                  P(ctypes.c_int), P(ctypes.c_int)]
    return lib


def _ref_data(path, V, N):
    out = np.empty((V + 1) * N, np.float64)
    _ref().ref_load_data(os.fsencode(path), V, N, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out.reshape(V + 1, N)


def _ref_gen(path):
    lib = _ref()
    E, T = ctypes.c_int(), ctypes.c_longlong()
    lib.ref_parse_gen(os.fsencode(path), ctypes.byref(E), ctypes.byref(T), None, None, None,
                      None, None)
    tok = np.empty(T.value, np.int32)
    val = np.empty(T.value, np.float64)
    off = np.empty(E.value + 1, np.int64)
    nv = np.empty(E.value, np.int32)
    nd = np.empty(E.value, np.int32)
    P = ctypes.POINTER
    lib.ref_parse_gen(os.fsencode(path), ctypes.byref(E), ctypes.byref(T),
                      tok.ctypes.data_as(P(ctypes.c_int)), val.ctypes.data_as(P(ctypes.c_double)),
                      off.ctypes.data_as(P(ctypes.c_longlong)), nv.ctypes.data_as(P(ctypes.c_int)),
                      nd.ctypes.data_as(P(ctypes.c_int)))
    return tok, val, off, nv, nd


@needs_ref
def test_shared_data_matches_reference_reader(tmp_path):
    rng = np.random.default_rng(1)
    V, N = 4, 30_011
    X = rng.standard_normal((V + 1, N)) * np.exp(rng.uniform(-30, 30, (V + 1, N)))
    X[0, :10] = [0.0, -0.0, 1e-320, 3.4e38, 1e39, -1e39, 1.5, 2.5, 7.0, -7.0]
    p = tmp_path / "shared_data.txt"
    with open(p, "w") as f:  # mixed separators, signs and exponents, CRLF, blank tail
        for j in range(N):
            fields = [repr(float(x)) if (j + v) % 3 else f"{x:+.17e}" for v, x in enumerate(X[:, j])]
            sep = "\t" if j % 7 == 0 else "  " if j % 5 == 0 else " "
            f.write(sep.join(fields) + ("\r\n" if j % 11 == 0 else "\n"))
        f.write("\n\n")
    want = _ref_data(str(p), V, N).astype(np.float32)
    for threads in (1, 3, 0):
        got = formats.load_shared_data(str(p), V, threads=threads)
        assert got.shape == (V + 1, N)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    got = formats.load_shared_data(str(p), V, num_dps=1000)
    assert np.array_equal(got.view(np.uint32), want[:, :1000].view(np.uint32))
    assert np.array_equal(formats.read_shared_data(str(p), V).astype(np.float32).view(np.uint32),
                          want.view(np.uint32))


def test_shared_data_malformed_line_is_rejected(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("1 2 3\n4 5\n7 8 9\n")
    with pytest.raises(SrError):
        formats.load_shared_data(str(p), 2)
    p.write_text("1 2 3\n4 5 6 7\n")
    with pytest.raises(SrError):
        formats.load_shared_data(str(p), 2)
    with pytest.raises(SrError):
        formats.load_shared_data(str(tmp_path / "missing.txt"), 2)


@needs_ref
def test_population_matches_reference_reader(tmp_path):
    w = synth.batched_workload(seed=5, E=700, N=1000)
    p = tmp_path / "gen_3.txt"
    formats.write_gen_file(str(p), w.population, 5, 1000, "shared_data.txt")
    tok, val, off, nv, nd = _ref_gen(str(p))
    for threads in (1, 4, 0):
        pop, nv2, nd2, name = formats.load_population(str(p), threads=threads)
        assert np.array_equal(pop.tokens, tok) and np.array_equal(pop.offsets, off)
        assert np.array_equal(pop.values.view(np.uint64), val.view(np.uint64))
        assert np.array_equal(nv2, nv) and np.array_equal(nd2, nd)
        assert name == "shared_data.txt"
    q = formats.read_gen_file(str(p))[0]
    assert np.array_equal(q.values.view(np.uint64), val.view(np.uint64))


def test_population_malformed_is_rejected(tmp_path):
    p = tmp_path / "gen_bad.txt"
    p.write_text("2\n1 10 3\n1 -1 -1\n0 0 1\nd.txt\n")  # second expression missing
    with pytest.raises(SrError):
        formats.load_population(str(p))
    p.write_text("1\n1 10 3\n1 -1\n0 0 1\nd.txt\n")  # too few tokens
    with pytest.raises(SrError):
        formats.load_population(str(p))
