"""Host-side lifetime rules of the Python mirror (no GPU): a native handle is
destroyed only after every object created on it, whatever order the
finalizers of a reference cycle run in."""
import gc


def _classes(sb):
    from sequoia_boost_b200.api import _Native
    log = []

    class Parent(_Native):
        def __init__(self, name):
            self.h = name

        def _free(self):
            log.append(self.h)

    class Child(_Native):
        def __init__(self, name, *parents):
            self.h = name
            self._adopt(*parents)

        def _free(self):
            log.append(self.h)

    return Parent, Child, log


def test_parent_finalized_first_waits_for_children(sb):
    Parent, Child, log = _classes(sb)
    ctx = Parent("ctx")
    model = Child("model", ctx)
    server = Child("server", ctx, model)
    # the finalizers of a collected cycle may run parent-first
    ctx.__del__()
    model.__del__()
    assert log == []
    server.__del__()
    assert log == ["server", "model", "ctx"]


def test_cycle_collected_by_gc_frees_children_first(sb):
    Parent, Child, log = _classes(sb)
    ctx = Parent("ctx")
    model = Child("model", ctx)
    ctx.back = model  # a reference cycle: ctx <-> model
    model.self_ref = model
    del ctx, model
    gc.collect()
    assert log == ["model", "ctx"]


def test_close_then_finalize_frees_once(sb):
    Parent, Child, log = _classes(sb)
    ctx = Parent("ctx")
    s = Child("server", ctx)
    s._released = True
    s._drop()
    s.__del__()
    assert log == ["server"]
    ctx.__del__()
    assert log == ["server", "ctx"]
