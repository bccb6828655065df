"""CPU checks of the boundary: the C-ABI library exists, loads, and exports
every symbol include/alfa.h declares; config marshalling; no compute."""
import ctypes
import os

import pytest

from jax_alfa_b200 import _lib, cases


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _lib.exported_symbols()
    assert len(declared) >= 40
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_signature_table_covers_header():
    declared = set(_lib.exported_symbols())
    bound = set(_lib.SIGNATURES) | {"alfa_create", "alfa_destroy", "alfa_last_error",
                                    "alfa_set_stream", "alfa_get_derived", "alfa_get_precision",
                                    "alfa_workspace_bytes", "alfa_get_diag",
                                    "alfa_launch_count", "alfa_time_kernel", "alfa_autotune",
                                    "alfa_set_line_variant", "alfa_tc_line_apply", "alfa_set_tc_spin_limit",
                                    "alfa_PlanarMean_noalloc", "alfa_checkpoint_doubles",
                                    "alfa_ensemble_create", "alfa_ensemble_step",
                                    "alfa_ensemble_sync", "alfa_ensemble_set_stream",
                                    "alfa_ensemble_error",
                                    "alfa_ensemble_destroy", "alfa_mlp_create",
                                    "alfa_mlp_destroy", "alfa_mlp_collect", "alfa_mlp_train",
                                    "alfa_mlp_loss_grad", "alfa_mlp_get_params",
                                    "alfa_mlp_set_params", "alfa_mlp_features",
                                    "alfa_mlp_infer", "alfa_step_learned"}
    assert declared <= bound, declared - bound


def test_config_struct_carries_every_case_option():
    from jax_alfa_b200.api import CONFIG_KEYS
    for make in cases.CASES.values():
        cfg = make()
        # precision follows the reference's use_double_precision switch
        missing = [k for k in CONFIG_KEYS if k not in cfg and k != "precision"]
        assert not missing, missing


def test_precision_follows_the_reference_switch():
    from jax_alfa_b200.api import make_config
    assert make_config(cases.neutral()).precision == _lib.FP64
    assert make_config(cases.neutral(use_double_precision=False)).precision == _lib.FP32
    assert make_config(cases.neutral(precision="mixed")).precision == _lib.MIXED
    assert make_config(cases.neutral(precision="fp32")).precision == _lib.FP32


def test_create_rejects_unknown_precision_without_gpu():
    from jax_alfa_b200.api import make_config
    lib = _lib.load()
    c = make_config(cases.neutral())
    c.precision = 7
    ctx = ctypes.c_void_p()
    assert lib.alfa_create(ctypes.byref(c), ctypes.byref(ctx)) == -1
    assert b"precision" in lib.alfa_last_error(None)


def test_create_rejects_bad_config_without_gpu():
    """alfa_create validates the configuration before touching the device."""
    from jax_alfa_b200.api import make_config
    lib = _lib.load()
    cfg = cases.neutral(30, 32, 32)   # nx = 30 = 2*3*5: radix 5 unsupported
    ctx = ctypes.c_void_p()
    rc = lib.alfa_create(ctypes.byref(make_config(cfg)), ctypes.byref(ctx))
    assert rc == -1
    assert b"2^a 3^b" in lib.alfa_last_error(None)
    cfg = cases.neutral(32, 32, 32, optSgs=5)  # STABSM: its modules are not in the reference
    rc = lib.alfa_create(ctypes.byref(make_config(cfg)), ctypes.byref(ctx))
    assert rc == -1 and b"optSgs" in lib.alfa_last_error(None)


def test_product_path_has_no_oracle_dependency():
    import jax_alfa_b200
    root = os.path.dirname(jax_alfa_b200.__file__)
    for dirpath, _, files in os.walk(root):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh")):
                with open(os.path.join(dirpath, f)) as fh:
                    text = fh.read()
                assert "from oracle" not in text and "import oracle" not in text, f
