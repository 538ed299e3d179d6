"""The C ABI library: it builds for sm_100a, loads without a GPU and exports
every symbol include/nhflood.h declares (no compute calls here)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope='module')
def library_path():
    from nhflood.build import build
    return build()


def declared_symbols():
    text = (ROOT / 'include' / 'nhflood.h').read_text()
    return sorted(set(re.findall(r'\b(nhf_[a-z_]+)\s*\(', text)))


def test_header_declares_the_bound_functions():
    from nhflood.native import exported_symbols
    assert sorted(exported_symbols()) == declared_symbols()


def test_library_exports_every_declared_symbol(library_path):
    out = subprocess.run(['nm', '-D', '--defined-only', str(library_path)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_without_a_gpu(library_path):
    lib = ctypes.CDLL(str(library_path))
    lib.nhf_version.restype = ctypes.c_char_p
    assert b'sm_100a' in lib.nhf_version()
    lib.nhf_last_error.restype = ctypes.c_char_p
    lib.nhf_last_error.argtypes = [ctypes.c_void_p]
    assert lib.nhf_last_error(None) == b''


def test_create_rejects_bad_arguments_without_touching_the_device(library_path):
    from nhflood.native import NhfMesh, NhfParams, library
    lib = library(library_path)
    handle = ctypes.c_void_p()
    mesh = NhfMesh()
    mesh.e_num, mesh.s_num = 3, 5
    params = NhfParams(9.81, .5, 1., .02, 1e-4, 65)  # batch above 64
    rc = lib.nhf_create(ctypes.byref(mesh), ctypes.byref(params), None, ctypes.byref(handle))
    assert rc == -1 and b'batch_size' in lib.nhf_last_error(None)
    params = NhfParams(9.81, .5, .7, .02, 1e-4, 32)  # theta < 1 without open-face fractions
    rc = lib.nhf_create(ctypes.byref(mesh), ctypes.byref(params), None, ctypes.byref(handle))
    assert rc == -1 and b'open_face' in lib.nhf_last_error(None)
    assert not handle.value


def test_kernels_compile_without_spills():
    """ptxas resource report for the step kernels (sm_100a)."""
    from nhflood.build import ARCH, CSRC, INCLUDE, nvcc
    out = subprocess.run([nvcc(), *ARCH, '-O3', '--fmad=false', '-std=c++17', '-Xptxas', '-v', '-c',
                          f'-I{INCLUDE}', '-o', '/dev/null', str(CSRC / 'nhf_step.cu')],
                         capture_output=True, text=True, check=True).stderr
    spills = [int(m) for m in re.findall(r'(\d+) bytes spill stores', out)]
    assert spills and max(spills) == 0, out


def test_fp64_build_exports_the_single_mesh_entry_points(library_path):
    """libnhflood_f64.so: the multi-pass step with nhf_real = double."""
    from nhflood.build import LIBRARY_F64
    from nhflood.native import exported_symbols, library
    out = subprocess.run(['nm', '-D', '--defined-only', str(LIBRARY_F64)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    single = [s for s in exported_symbols() if not s.startswith(('nhf_ensemble', 'nhf_cfl_noalloc'))]
    assert not [s for s in single if s not in exported]
    lib = library(precision='f64')
    assert lib.nhf_real_bytes() == 8 and b'FP64' in lib.nhf_version()
    assert library().nhf_real_bytes() == 4
