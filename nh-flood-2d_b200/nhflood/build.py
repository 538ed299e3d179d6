"""Build the sm_100a step libraries in-tree: nhflood/_lib/libnhflood.so
(every step form, F32 physics) and nhflood/_lib/libnhflood_f64.so (the
multi-pass step compiled with -DNHF_REAL_DOUBLE: the same kernels with F64
physics, for the precision study).

Flags: --fmad=false keeps the reference's F32 operation sequence (no
multiply-add contraction), which the CPU restatement reproduces bit for bit;
IEEE division and square root are nvcc's defaults and stay on.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = ROOT / 'csrc'
LIBDIR = PACKAGE / '_lib'
LIBRARY = LIBDIR / 'libnhflood.so'
LIBRARY_F64 = LIBDIR / 'libnhflood_f64.so'
F64_SOURCES = ('nhf_step.cu',)  # the FP64 build: the multi-pass step only
INCLUDE = ROOT.parent / 'include'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc() -> str:
    found = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(found).exists():
        raise RuntimeError('nvcc not found; the CUDA toolkit is required to build libnhflood.so')
    return found


def sources() -> list[Path]:
    return sorted(CSRC.glob('*.cu'))


def needs_build(library: Path = LIBRARY) -> bool:
    if not library.exists():
        return True
    stamp = library.stat().st_mtime
    deps = sources() + sorted(CSRC.glob('*.cuh')) + sorted(INCLUDE.glob('*.h'))
    return any(p.stat().st_mtime > stamp for p in deps)


PREP_LIBRARY = LIBDIR / 'libnhfprep.so'


def host_sources() -> list[Path]:
    return sorted((CSRC / 'host').glob('*.cpp'))


def build_host(verbose: bool = False, force: bool = False) -> Path:
    """The host-only preprocessing library (g++, no CUDA): libnhfprep.so."""
    deps = host_sources() + [INCLUDE / 'nhf_prep.h']
    if not force and PREP_LIBRARY.exists() and all(p.stat().st_mtime <= PREP_LIBRARY.stat().st_mtime for p in deps):
        return PREP_LIBRARY
    LIBDIR.mkdir(exist_ok=True)
    tmp = LIBDIR / f'.libnhfprep.{os.getpid()}.so'
    cmd = [shutil.which('g++') or 'g++', '-O2', '-std=c++17', '-fPIC', '-shared', f'-I{INCLUDE}', '-o', str(tmp),
           *map(str, host_sources())]
    if verbose:
        print(' '.join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, PREP_LIBRARY)
    return PREP_LIBRARY


def _nvcc_shared(library: Path, files, defines=(), verbose=False) -> None:
    LIBDIR.mkdir(exist_ok=True)
    tmp = LIBDIR / f'.{library.stem}.{os.getpid()}.so'
    cmd = [nvcc(), *ARCH, '-lineinfo', '-O3', '--fmad=false', '-std=c++17', '-Xcompiler', '-fPIC',
           *defines, '-shared', f'-I{INCLUDE}', '-o', str(tmp), *map(str, files)]
    if verbose:
        print(' '.join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, library)


def build(verbose: bool = False, force: bool = False) -> Path:
    build_host(verbose, force)
    if force or needs_build(LIBRARY):
        _nvcc_shared(LIBRARY, sources(), verbose=verbose)
    if force or needs_build(LIBRARY_F64):
        _nvcc_shared(LIBRARY_F64, [CSRC / f for f in F64_SOURCES], ['-DNHF_REAL_DOUBLE'], verbose)
    return LIBRARY


if __name__ == '__main__':
    print(build(verbose=True, force='--force' in sys.argv))
