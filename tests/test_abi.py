"""The C ABI without a GPU: the library loads, exports every symbol that
include/sb_gpu.h declares, its structs match the header, host-side parameter
validation mirrors TrainingParams::validate, and compute entry points fail
loudly (SB_ERR_NO_DEVICE) instead of falling back to the CPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "sb_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(sb):
    from sequoia_boost_b200 import _abi
    lib = _abi.lib()
    syms = header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) == set(_abi.SIGNATURES), set(syms) ^ set(_abi.SIGNATURES)


def test_struct_layouts_match_oracle_view(sb, orc):
    from sequoia_boost_b200 import _abi
    import sb_pyoracle as po
    for a, b in [(_abi.SbNode, po.Node), (_abi.SbTrainParams, po.Params),
                 (_abi.SbModelView, po.ModelView), (_abi.SbGradPair, po.GradPair),
                 (_abi.SbGradStats, po.GradStats)]:
        assert ctypes.sizeof(a) == ctypes.sizeof(b)
        assert [f[0] for f in a._fields_] == [f[0] for f in b._fields_]
        for (n1, _), (n2, _) in zip(a._fields_, b._fields_):
            assert getattr(a, n1).offset == getattr(b, n2).offset
    assert ctypes.sizeof(_abi.SbNode) == 40
    assert ctypes.sizeof(_abi.SbTrainParams) == 8 * 16 + 4 * 12


def test_defaults_match_reference(sb):
    from sequoia_boost_b200 import _abi
    p = _abi.SbTrainParams()
    _abi.lib().sb_train_params_default(ctypes.byref(p))
    # config/params.rs:153-186
    assert (p.eta, p.max_depth, p.min_child_weight, p.lambda_, p.max_bin, p.subsample) == \
        (0.3, 6, 1.0, 1.0, 256, 1.0)
    assert p.has_base_score == 0 and p.grow_policy == 0 and p.objective == 0


@pytest.mark.parametrize("field,value,ok", [
    ("eta", 0.0, False), ("eta", -1.0, False), ("gamma", -1.0, False), ("subsample", 0.0, False),
    ("subsample", 1.5, False), ("colsample_bytree", 1.1, False), ("max_bin", 1, False),
    ("lambda_", float("nan"), False), ("scale_pos_weight", 0.0, False), ("eta", 0.1, True),
])
def test_validate_matches_reference_and_oracle(sb, orc, field, value, ok):
    p = sb.TrainingParams()
    setattr(p, field, value)
    if ok:
        p.validate()
    else:
        with pytest.raises(sb.SbError):
            p.validate()
    assert orc.validate(p) == ok


def test_lossguide_needs_a_bound(sb, orc):
    p = sb.TrainingParams(grow_policy="lossguide", max_leaves=0, max_depth=0)
    with pytest.raises(sb.SbError):
        p.validate()
    assert not orc.validate(p)


def test_multiclass_needs_num_class(sb):
    with pytest.raises(sb.SbError):
        sb.TrainingParams(objective="multi:softprob", num_class=1).validate()
    with pytest.raises(sb.SbError):
        sb.TrainingParams(objective="nope:whatever").validate()


def test_no_cpu_fallback_without_gpu(sb):
    from sequoia_boost_b200 import _abi
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    rc = _abi.lib().sb_ctx_create(0, ctypes.byref(h))
    assert rc == _abi.SB_ERR_NO_DEVICE
    assert b"no CUDA device" in _abi.lib().sb_last_error()
    with pytest.raises(sb.SbError):
        sb.Context(0)


def test_null_arguments_are_rejected(sb):
    from sequoia_boost_b200 import _abi
    lib = _abi.lib()
    assert lib.sb_ctx_create(0, None) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_ghist_info(None, None, None, None) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_model_export_sizes(None, None, None, None) == _abi.SB_ERR_INVALID_ARG
    assert lib.sb_booster_update(None, 1) == _abi.SB_ERR_INVALID_ARG


def test_model_view_roundtrip_host_only(sb):
    """sb_model_create / export keep a host copy: no device needed."""
    from sequoia_boost_b200 import _abi
    from sequoia_boost_b200.api import NODE_DTYPE
    nodes = np.zeros(3, NODE_DTYPE)
    nodes["left"] = [1, -1, -1]
    nodes["right"] = [2, -1, -1]
    nodes["split_cond"][0] = 0.5
    nodes["leaf_value"][1:] = [-1.0, 2.0]
    off = np.array([0, 3], np.int64)
    coff = np.array([0, 0], np.int64)
    cats = np.zeros(1, np.uint32)
    v = _abi.SbModelView()
    v.tree_node_offset = off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    v.nodes = nodes.ctypes.data_as(ctypes.POINTER(_abi.SbNode))
    v.tree_cat_offset = coff.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    v.categories = cats.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    v.n_trees, v.num_class, v.n_features, v.base_score = 1, 0, 1, 0.25
    # a context is required; without a GPU the model handle cannot be made
    h = ctypes.c_void_p()
    rc = _abi.lib().sb_model_create(None, ctypes.byref(v), ctypes.byref(h))
    assert rc == _abi.SB_ERR_INVALID_ARG
