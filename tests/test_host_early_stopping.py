"""train_impl's early-stopping rule (learner/train.rs:264-271, 350-377) as
the host mirror runs it; no GPU."""


def test_stops_after_patience_rounds_without_strict_improvement(sb):
    from sequoia_boost_b200.api import EarlyStopping
    es = EarlyStopping(3)
    vals = [1.0, 0.8, 0.7, 0.7, 0.75, 0.71]  # 0.7 repeated is not an improvement
    stops = [es.update(r, v) for r, v in enumerate(vals)]
    assert stops == [False, False, False, False, False, True]
    assert es.best_iteration == 2


def test_no_patience_never_stops(sb):
    from sequoia_boost_b200.api import EarlyStopping
    es = EarlyStopping(None)
    assert not any(es.update(r, 1.0) for r in range(50))
    assert es.best_iteration is None


def test_maximized_metric(sb):
    from sequoia_boost_b200.api import EarlyStopping
    es = EarlyStopping(2, maximize=True)
    stops = [es.update(r, v) for r, v in enumerate([0.5, 0.6, 0.6, 0.55])]
    assert stops == [False, False, False, True] and es.best_iteration == 1
