"""The C ABI library builds, loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dada2_b200.h")


def declared_symbols():
    text = open(HEADER, encoding="utf-8").read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dgpu_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_symbols()
    for required in ("dgpu_ctx_create", "dgpu_upload_raws", "dgpu_compare", "dgpu_compare_store",
                     "dgpu_dada", "dgpu_dada_batch", "dgpu_ctx_destroy", "dgpu_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from dada2_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        import importlib.util

        spec = importlib.util.spec_from_file_location("dgpu_build", os.path.join(ROOT, "dada2-rs_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_errors_are_reported_without_a_device():
    from dada2_b200 import _lib

    L = _lib.lib()
    n = ctypes.c_int(-1)
    rc = L.dgpu_device_count(ctypes.byref(n))
    assert rc in (0, _lib.DGPU_E_CUDA)
    # a null argument is rejected before any CUDA call
    rc = L.dgpu_result_sizes(None, None)
    assert rc == _lib.DGPU_E_INVALID
    assert b"null" in L.dgpu_last_error()


def test_gpu_entry_points_fail_loudly_without_a_device():
    import numpy as np

    import dada2_b200 as D

    if D.device_count() > 0:
        pytest.skip("a GPU is present; covered by the gpu tests")
    with pytest.raises(D.DgpuError):
        D.dada_uniques(["ACGTACGTAC"], [3], np.full(16, 0.01), 1)


def test_sharded_run_keeps_its_ranks_in_step_without_a_device():
    """dgpu_dada_sharded: argument errors return before any exchange; a rank
    that cannot prepare (no device here) still takes part in the setup
    exchange, once, reporting its error, so its peers stop there too."""
    import numpy as np

    import dada2_b200 as D

    if D.device_count() > 0:
        pytest.skip("a GPU is present; covered by the gpu tests")
    calls = []

    def gather(block):
        calls.append(block.size)
        return np.concatenate([block, block])

    args = (["ACGTACGTAC"], [3], np.full(16, 0.01), 1)
    with pytest.raises(D.InvalidInput, match="rank out of range"):
        D.dada_uniques_sharded(*args, rank=2, world=2, gather=gather)
    assert calls == []
    with pytest.raises(D.DgpuError):
        D.dada_uniques_sharded(*args, rank=0, world=2, gather=gather)
    assert calls == [56]


def test_service_lifecycle_without_a_device():
    """Without a GPU the service's worker fails every request with a CUDA
    error instead of hanging, and destroy returns."""
    import numpy as np

    import dada2_b200 as D

    if D.device_count() > 0:
        pytest.skip("a GPU is present; covered by the gpu tests")
    with pytest.raises(D.DgpuError):  # a zero budget queries the device
        D.DenoiseService(np.full(16, 0.01), 1)
    svc = D.DenoiseService(np.full(16, 0.01), 1, hbm_budget=1 << 30)
    try:
        t = None
        try:
            t = svc.submit(["ACGTACGTAC"], [3])
        except D.DgpuError:
            pass  # the worker already stopped on the missing device
        if t is not None:
            with pytest.raises(D.DgpuError, match="cudaSetDevice"):
                svc.wait(t)
    finally:
        svc.close()


def test_library_calc_pA_matches_the_oracle_bit_for_bit():
    """The host p-value (calc_pA, src/pval.rs:208-241) the library exports is
    the oracle's to the last bit, over both gamma branches, the log-space
    fallback and the conditioning (no GPU needed)."""
    import numpy as np

    import dada2_b200 as D
    from oracle import oracle as O

    for k in (1, 2, 3, 5, 10, 40, 200, 3000):
        for le in np.linspace(-17, 4, 85):
            e = float(10.0 ** le)
            for prior in (False, True):
                a, b = D.calc_pA(k, e, prior), O.calc_pA(k, e, prior)
                assert np.float64(a).tobytes() == np.float64(b).tobytes(), (k, e, prior, a, b)
