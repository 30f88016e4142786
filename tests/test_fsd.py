"""The .fsd / .frs reader and writer: WTDATA's record framing and order
(src/fasolt/Faslt_io_nowin.f90:185-299) and RDDATA's reading of it."""
import struct

import numpy as np

from cpfem_code_b200 import fsd, generator


def _fields(p):
    return ("le", "lt", "nd", "np_", "ln", "lg", "ib", "x", "dx", "fc", "eps", "dep", "st", "ep", "ds",
            "de", "rt", "dr", "sv", "dsv", "nss", "e", "ssang", "ab", "an", "ampar", "smatrx", "tiem",
            "x_spec", "f_spec")


def test_roundtrip_real8(tmp_path):
    p = generator.mixed_config(n=2, ninc=3)
    p.st[:] = np.random.default_rng(1).standard_normal(p.st.shape)
    path = str(tmp_path / "a.frs")
    fsd.write(path, p, first_record=2, real_bytes=8)
    q, first = fsd.read(path, real_bytes=8)
    assert first == 2
    for k in _fields(p):
        np.testing.assert_array_equal(getattr(q, k), getattr(p, k), err_msg=k)
    assert (q.nlmnt, q.nnod, q.ngps, q.nsv, q.nmpar, q.nxs, q.nfs) == (p.nlmnt, p.nnod, p.ngps, p.nsv, p.nmpar, p.nxs, p.nfs)
    assert q.twinlim == p.twinlim and q.twinprob == p.twinprob


def test_roundtrip_20_node_bricks(tmp_path):
    """20-node, 8-Gauss-point bricks (the element type of the reference's
    sample input) keep their 20 node and 8 GP ids per element."""
    p = generator.structured_cube(n=(2, 1, 2), ninc=2, nodes=20)
    path = str(tmp_path / "b.fsd")
    fsd.write(path, p, real_bytes=8)
    q, _ = fsd.read(path, real_bytes=8)
    for k in _fields(p):
        np.testing.assert_array_equal(getattr(q, k), getattr(p, k), err_msg=k)
    assert q.ln.shape == (p.nlmnt, 20) and q.lg.shape == (p.nlmnt, 8)


def test_roundtrip_real4_rounds_to_float32(tmp_path):
    p = generator.structured_cube(n=(2, 1, 1), ninc=2)
    path = str(tmp_path / "a.fsd")
    fsd.write(path, p)
    q, first = fsd.read(path)
    assert first == p.ninc1
    np.testing.assert_array_equal(q.e, p.e.astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(q.sv, p.sv.astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(q.ln, p.ln)


def test_record_framing(tmp_path):
    p = generator.structured_cube(n=(1, 1, 1), ninc=1)
    path = str(tmp_path / "b.fsd")
    fsd.write(path, p)
    b = open(path, "rb").read()
    # record 1: ninc1 (one INTEGER(4)), framed by 4-byte lengths
    assert struct.unpack_from("<iii", b, 0) == (4, 1, 4)
    # record 2: nlmnt, nnod, ngps, nsv
    assert struct.unpack_from("<i4ii", b, 12) == (16, 1, 8, 1, 15, 16)
    # record 3: le, lt, nd, np of element 1
    assert struct.unpack_from("<i4ii", b, 36) == (16, 1, 12, 8, 1, 16)
    # record 4: the 8 node ids
    assert struct.unpack_from("<i8ii", b, 60) == (32, 1, 2, 3, 4, 5, 6, 7, 8, 32)
