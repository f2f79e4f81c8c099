"""CPU-side checks of the C ABI: the in-tree library loads, exports every
function include/amica_b200.h declares, and behaves on the paths that need no
GPU (defaults, status strings, argument validation).  No compute calls."""
import ctypes as C
import os
import re

import pytest

from cudamica_b200 import engine as E

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "amica_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(amica_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(E.LIB_PATH):
        from cudamica_b200 import build
        build.build()
    return E.lib()


def test_header_symbols_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(E.EXPORTED) | {"amica_stats_len"}


def test_default_cfg_matches_reference_defaults(lib):
    cfg = E.default_cfg()
    # include/config.h:46-83 of the reference
    assert (cfg.nsdm, cfg.nmmodels, cfg.maxiter, cfg.do_sphere, cfg.block_size) == (3, 1, 200, 1, 5000)
    assert (cfg.do_newton, cfg.newt_start_iter, cfg.rho_start_iter, cfg.maxdec) == (1, 50, 1, 3)
    assert (cfg.lrate0, cfg.lratemax, cfg.lnatrate, cfg.lratefact) == (0.1, 1.0, 0.1, 0.5)
    assert (cfg.rho0, cfg.rholrate, cfg.rhomin, cfg.rhomax) == (1.5, 0.1, 1.0, 2.0)


def test_status_strings(lib):
    assert lib.amica_status_string(0) == b"Success!"
    assert lib.amica_status_string(-5) == b"No file"
    assert b"singular" in lib.amica_status_string(-22)
    assert lib.amica_status_string(12345) == b"Unknown error"


def test_stats_len(lib):
    assert lib.amica_stats_len(32, 1, 3) == 1 + (1 + 64 + 1024 + 7 * 96)


def test_invalid_arguments_rejected(lib):
    ctx = C.c_void_p()
    assert lib.amica_create(None, C.byref(ctx)) == -3
    cfg = E.default_cfg(nchannels=1, nsamples=10)
    assert lib.amica_create(C.byref(cfg), C.byref(ctx)) == -3
    cfg = E.default_cfg(nchannels=8, nsamples=100, nmmodels=9)
    assert lib.amica_create(C.byref(cfg), C.byref(ctx)) == -25
    assert lib.amica_em_step(None, None) == -3
    assert lib.amica_destroy(None) == 0


def test_create_without_gpu_reports_no_device(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    ctx = C.c_void_p()
    cfg = E.default_cfg(nchannels=8, nsamples=100)
    assert lib.amica_create(C.byref(cfg), C.byref(ctx)) == -26


def test_noalloc_argument_checks(lib):
    # argument checks come before any device call, so they hold without a GPU;
    # dummy non-null pointers are never dereferenced on these paths
    f = E.estep_stats_noalloc
    with pytest.raises(E.AmicaError) as ei:
        # keep = NULL means every sample counts: nkeep must then be T
        f(1, 32, 32, 1000, 1, 3, 1, 1, 1, 1, 1, 1, 1, 0.0, 1, keep_ptr=0, nkeep=900)
    assert ei.value.code == -3
    with pytest.raises(E.AmicaError) as ei:
        f(1, 64, 32, 1000, 1, 3, 1, 1, 1, 1, 1, 1, 1, 0.0, 1)     # ldx must be 32 for n = 32
    assert ei.value.code == -3
