"""The flat precision module of the reference (dense_evolution/config.py:29-62):
set_precision / ensure_x64 / with_x64 and the default they give to
constructors that are not told a precision."""
import importlib


def test_config_module_semantics():
    cfg = importlib.import_module('dense_evolution.config')
    saved = (cfg._float64, cfg._explicit)
    cfg._float64, cfg._explicit = True, False
    assert cfg.float64_enabled() and not cfg.default_use_float32(None)
    assert cfg.default_use_float32(True) and not cfg.default_use_float32(False)
    cfg.ensure_x64()
    assert cfg.float64_enabled()
    cfg.set_precision(False)
    cfg.ensure_x64()                      # an explicit choice sticks
    assert not cfg.float64_enabled() and cfg.default_use_float32(None)

    calls = []

    @cfg.with_x64
    def f(x):
        calls.append(cfg.float64_enabled())
        return x + 1

    assert f(1) == 2 and calls == [False]
    assert f.__name__ == 'f'
    cfg.set_precision(True)
    assert cfg.float64_enabled()
    cfg._float64, cfg._explicit = saved   # back to the process default for later tests


def test_package_exports_config():
    import dense_evolution as de
    assert de.set_precision is de.config.set_precision
