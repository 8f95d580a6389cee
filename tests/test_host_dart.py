"""DART's dropout draw (train.rs:397-425) as the host mirror makes it; no GPU."""


def test_dropout_rules(sb):
    from sequoia_boost_b200.api import dart_dropout
    assert dart_dropout(1, 0, 0, 0.5, 0.0) == []           # no trees yet
    assert dart_dropout(1, 3, 10, 0.5, 1.0) == []          # always skipped
    one = dart_dropout(1, 3, 10, 0.0, 0.0)                  # nothing drawn: one tree is dropped
    assert len(one) == 1 and 0 <= one[0] < 10
    assert dart_dropout(1, 3, 10, 1.0, 0.0) == list(range(10))
    assert dart_dropout(7, 5, 50, 0.3, 0.0) == dart_dropout(7, 5, 50, 0.3, 0.0)  # deterministic
    sizes = [len(dart_dropout(7, r, 1000, 0.1, 0.0)) for r in range(40)]
    assert 80 < sum(sizes) / len(sizes) < 120               # about rate_drop of the trees
    skipped = sum(dart_dropout(9, r, 20, 0.5, 0.25) == [] for r in range(400))
    assert 70 < skipped < 130                               # about skip_drop of the rounds


def test_params_validation(sb):
    import pytest
    with pytest.raises(sb.SbError):
        sb.TrainingParams(booster="dart", rate_drop=1.5).validate()
    with pytest.raises(sb.SbError):
        sb.TrainingParams(booster="gblinear").validate()
    sb.TrainingParams(booster="dart", rate_drop=0.1, skip_drop=0.5).validate()
