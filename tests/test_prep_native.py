"""The C++ NE/NS preprocessing (libnhfprep.so) builds exactly the tables of
the Python restatement of the reference's preprocessing: filtered cells
(bed -9999), dropped sides, renumbering, face CSR, topology, coordinates."""
import numpy as np
import pytest

from nhflood import preprocess as P
from nhflood.workloads import multires_quadtree, plain_uniform_256


def python_tables(ne_text: str, ns_text: str):
    ne, ns = P.filter_ne_ns(ne_text.splitlines(keepends=True), ns_text.splitlines(keepends=True))
    return P.build_ne_tables(ne), P.build_ns_tables(ns)


def assert_same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)


@pytest.fixture(scope='module')
def lib():
    from nhflood.build import build_host
    build_host()
    assert P.native_library() is not None
    return P.native_library()


@pytest.mark.parametrize('make', [lambda: plain_uniform_256(n=24).mesh,
                                  lambda: multires_quadtree(width=1000.0, duration=60).mesh])
def test_native_tables_equal_the_python_tables(tmp_path, lib, make):
    mesh = make()
    P.write_ne_ns(mesh, tmp_path / 'ne.txt', tmp_path / 'ns.txt')
    ne_text, ns_text = (tmp_path / 'ne.txt').read_text(), (tmp_path / 'ns.txt').read_text()
    # knock out a few cells (bed -9999) so filtering and renumbering matter
    lines = ne_text.splitlines()
    for k in range(3, len(lines), 37):
        f = lines[k].split(',')
        f[-2] = '-9999'
        lines[k] = ','.join(f)
    ne_text = '\n'.join(lines) + '\n'
    want_ne, want_ns = python_tables(ne_text, ns_text)
    got_ne, got_ns = P.native_tables(ne_text.encode(), ns_text.encode())
    assert len(got_ne['x']) < mesh.e_num  # cells were dropped
    assert_same(want_ne, got_ne)
    assert_same(want_ns, got_ns)


def test_malformed_text_is_rejected(lib):
    with pytest.raises(ValueError, match='NE line 1'):
        P.native_tables(b'1,1,1,x,1,1,2,3,4,5,5,0,10\n', b'')


def test_library_exports_every_declared_entry_point(lib):
    import re
    from nhflood.build import INCLUDE
    declared = re.findall(r'\b(nhp_[a-z_]+)\s*\(', (INCLUDE / 'nhf_prep.h').read_text())
    assert set(declared) == {'nhp_prepare', 'nhp_sizes', 'nhp_copy_cells', 'nhp_copy_sides', 'nhp_free', 'nhp_error'}
    for name in declared:
        assert hasattr(lib, name)
