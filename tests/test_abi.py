"""The C-ABI library on the CPU side: it loads without a GPU, exports every symbol include/chaoslab_b200.h
declares, its structs match the ctypes mirror, every compiled menu key passes `cl_b200_check`, and ill-formed runs
are rejected with the reference's argument errors before any device work."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from chaos_b200 import _abi
from chaos_b200._lib import LIB_PATH, last_error, lib, menu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "chaoslab_b200.h")).read()
    declared = set(re.findall(r"CL_API\s+[\w\s\*]+?\b(cl_b200_\w+)\s*\(", hdr))
    assert declared == set(_abi.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (cl_b200_\w+)", out))
    assert declared <= exported, declared - exported
    L = lib()
    for name in declared:
        assert getattr(L, name) is not None


def test_struct_layout_matches_header():
    # compile a probe of the header's sizes/offsets with the host C compiler and compare with ctypes
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "chaoslab_b200.h"
int main(void){
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(cl_system), sizeof(cl_reducer), sizeof(cl_frame), sizeof(cl_run),
         sizeof(cl_buffers), sizeof(cl_prov), sizeof(cl_probe));
  printf("%zu %zu %zu %zu\n", offsetof(cl_run, sys), offsetof(cl_run, frames), offsetof(cl_run, orbit_base),
         offsetof(cl_system, A));
  printf("%zu %zu %zu\n", sizeof(cl_window), offsetof(cl_window, window), offsetof(cl_window, obs_b));
  return 0; }
'''
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "p.c")
        open(c, "w").write(src)
        exe = os.path.join(td, "p")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(v) for v in lines[0].split()]
    assert sizes == [C.sizeof(t) for t in (_abi.cl_system, _abi.cl_reducer, _abi.cl_frame, _abi.cl_run,
                                           _abi.cl_buffers, _abi.cl_prov, _abi.cl_probe)]
    offs = [int(v) for v in lines[1].split()]
    assert offs == [_abi.cl_run.sys.offset, _abi.cl_run.frames.offset, _abi.cl_run.orbit_base.offset,
                    _abi.cl_system.A.offset]
    assert [int(v) for v in lines[2].split()] == [C.sizeof(_abi.cl_window), _abi.cl_window.window.offset,
                                                  _abi.cl_window.obs_b.offset]


def _run_from_key(key: str) -> _abi.cl_run:
    m = re.match(r"s(\d+)d(\d+)p(\d+)\|(.*)", key)
    kind, d, p, rest = int(m[1]), int(m[2]), int(m[3]), m[4]
    wrapped = kind in (_abi.SYS_WRAPPED_STANDARD, _abi.SYS_WRAPPED_FROESCHLE, _abi.SYS_WRAPPED_CHAIN)
    r = _abi.cl_run(abi_version=_abi.ABI_VERSION, d=d, s=2 * d if wrapped else d, tau=1, N=10, n_frames=0,
                    precision=p)
    r.sys.kind = kind
    r.sys.n_sites = d // 2
    r.sys.gauss_maxiter = 50
    r.sys.dt = 0.01
    r.sys.n_stages = 2                      # a table method: the DKD leapfrog
    r.sys.stage_c[0] = r.sys.stage_c[1] = 0.5
    r.sys.stage_d[0] = 1.0
    for f, grp in enumerate(g for g in rest.split("|") if g):
        k, toks = grp.split(":")
        r.frames[f].k = int(k[1:])
        toks = [t for t in toks.split(",") if t]
        r.frames[f].n_reducers = len(toks)
        for i, t in enumerate(toks):
            rd = r.frames[f].reducers[i]
            if t.startswith("QR"):
                rd.kind, rd.alg, rd.orthogonality_tol = _abi.RED_QR, int(t[2:]), 8.0
            elif t == "BEN":
                rd.kind = _abi.RED_BENETTIN
            elif t == "SALI":
                rd.kind = _abi.RED_SALI
            elif t == "GALI":
                rd.kind = _abi.RED_GALI
            elif t.startswith("MEGNO"):
                rd.kind, rd.replace = _abi.RED_MEGNO, int(t[5:])
            elif t.startswith("FLI"):
                rd.kind, rd.replace = _abi.RED_FLI, int(t[3:])
        r.n_frames = f + 1
    return r


def test_every_menu_key_checks():
    keys = menu()
    assert len(keys) > 100 and len(set(keys)) == len(keys)
    L = lib()
    for key in keys:
        r = _run_from_key(key)
        assert L.cl_b200_check(C.byref(r)) == 0, (key, last_error())


def test_state_bytes_match_julia_layout():
    from chaos_b200 import GALI, MEGNO, SALI, FLI, Benettin, QRSpectrum, MGS
    from chaos_b200.reducers import chain_dtype
    assert chain_dtype((QRSpectrum(MGS()),), 2, 2).itemsize == 16 * 2 + 72
    assert chain_dtype((GALI(), SALI()), 4, 4).itemsize == 24 * 4 + 32 + 72
    assert chain_dtype((MEGNO(False), FLI(False), QRSpectrum(MGS())), 4, 2).itemsize == 200 + 96 + 104
    assert chain_dtype((Benettin(),), 2, 1).itemsize == 48


def test_argument_errors():
    from chaos_b200 import QRSpectrum, MGS, SALI, Benettin, StandardMap, propagate
    x0 = np.zeros((3, 2))
    with pytest.raises(ValueError, match="positive multiple of tau"):
        propagate(StandardMap(1.0), x0, 10, k=2, tau=3, reducers=(QRSpectrum(MGS()),))
    with pytest.raises(ValueError, match="k must be in 1:2"):
        propagate(StandardMap(1.0), x0, 10, k=3)
    with pytest.raises(ValueError, match="SALI needs k = 2"):
        propagate(StandardMap(1.0), x0, 10, k=1, reducers=(SALI(),))
    with pytest.raises(ValueError, match="Benettin needs k = 1"):
        propagate(StandardMap(1.0), x0, 10, k=2, reducers=(Benettin(),))
    with pytest.raises(ValueError, match="below the system dimension"):
        propagate(StandardMap(1.0), np.zeros((3, 1)), 10, k=1)
    with pytest.raises(ValueError, match="W0 needs one matrix per orbit"):
        propagate(StandardMap(1.0), x0, 10, k=2, W0=np.zeros((2, 2, 2)))
    with pytest.raises(ValueError, match="chunk must be positive"):
        propagate(StandardMap(1.0), x0, 10, k=2, chunk=0)


def test_unsupported_is_reason_3():
    from chaos_b200 import DeviceError, FroeschleMap, QRSpectrum, RGS, propagate
    with pytest.raises(DeviceError) as e:   # mixed-precision RGS on Froeschle k = 3 is not in the compiled menu
        propagate(FroeschleMap(1, 1, 0), np.zeros((2, 4)), 10, k=3, reducers=(QRSpectrum(RGS()),), precision="mixed")
    assert e.value.reason == 3


def test_variant_pinning_on_the_host():
    from chaos_b200 import FrameSpec as FS, Gauss, HenonHeilesFlow, IntegratorMap, MGS, QRSpectrum, StandardMap
    from chaos_b200.propagate import build_run
    lb = lib()
    g = build_run(IntegratorMap(Gauss(3), HenonHeilesFlow(), 0.01), 10, 1, [FS(2, (QRSpectrum(MGS()),))], "fp64", 0)
    assert lb.cl_b200_variants(C.byref(g)) == 0b1              # one register budget compiled for the Gauss step
    assert lb.cl_b200_set_variant(C.byref(g), 1) == 0 and lb.cl_b200_set_variant(C.byref(g), 0) == 0
    assert lb.cl_b200_set_variant(C.byref(g), 3) == _abi.EINVAL
    assert lb.cl_b200_set_variant(C.byref(g), 7) == _abi.EINVAL
    s = build_run(StandardMap(1.0), 10, 1, [FS(2, (QRSpectrum(MGS()),))], "fp64", 0)
    mask = lb.cl_b200_variants(C.byref(s))
    assert mask != 0 and lb.cl_b200_set_variant(C.byref(s), 1 + int(np.log2(mask & -mask))) == 0
    lb.cl_b200_set_variant(C.byref(s), 0)


def test_lattice_instances_offer_the_cooperative_variant():
    """Lattices with d >= 8 and one frame have the one-thread kernel (variant 1) and the cooperative form (variant
    8); d = 4 lattices and two-frame runs have no cooperative form."""
    from chaos_b200 import GALI, MGS, FrameSpec as FS, HouseholderQR, QRSpectrum, StandardMapChain
    from chaos_b200.propagate import build_run
    lb = lib()
    for sites in (4, 5, 8):
        for chain in ((QRSpectrum(HouseholderQR()),), (QRSpectrum(MGS()),), (GALI(),)):
            for prec in ("fp64", "mixed"):
                r = build_run(StandardMapChain(sites, 1.0, 0.05), 10, 1, [FS(8, chain)], prec, 0)
                assert lb.cl_b200_variants(C.byref(r)) == (1 | 1 << 7)
    r = build_run(StandardMapChain(2, 1.0, 0.05), 10, 1, [FS(4, (QRSpectrum(MGS()),))], "fp64", 0)
    assert lb.cl_b200_variants(C.byref(r)) == 1
    assert lb.cl_b200_set_variant(C.byref(r), 8) == _abi.EINVAL
