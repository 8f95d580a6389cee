"""sequoia-boost-b200: the B200 backend of sequoia-boost's hist training path.

A thin Python mirror of the reference crate's public API (crates/sequoia-boost/
src/lib.rs:86-97) over the C ABI in include/sb_gpu.h:

    TrainingParams   config/params.rs:76-373
    DMatrix          data/dmatrix.rs (dense f32 storage)
    train            learner/train.rs:107-113
    BoostedModel     learner/model.rs (predict_margin, predict, predict_leaf,
                     predict_contribs, predict_interactions, to/from_xgboost_json)
    xgboost_json     model/xgboost_json.rs (XGBoost JSON model import/export)
    GHistIndex       data/ghist.rs + data/quantile.rs (device-resident cuts/bins)
    GpuBackend       tree/hist/mod.rs:31-45 (HistogramBackend: build, subtract)
    HistTreeBuilder  tree/builder/hist.rs:98-202
    Booster          the device-resident state of train_impl's round loop
    objective_gradient  objective/mod.rs:58-69 (Objective::gradient)

All compute runs in libsb_gpu.so on an sm_100 GPU; there is no CPU fallback.
"""
from .api import (  # noqa: F401
    BoostedModel,
    Booster,
    Context,
    DMatrix,
    GHistIndex,
    GpuBackend,
    HistTreeBuilder,
    Monotone,
    Server,
    objective_gradient,
    TrainingParams,
    default_context,
    train,
    train_many,
    train_with_eval,
)
from ._abi import SbError  # noqa: F401

__all__ = [
    "BoostedModel", "Booster", "Context", "DMatrix", "GHistIndex", "GpuBackend",
    "HistTreeBuilder", "Monotone", "SbError", "Server", "TrainingParams", "default_context", "objective_gradient", "train", "train_many",
    "train_with_eval",
]
