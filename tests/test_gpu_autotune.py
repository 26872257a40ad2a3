"""The autotuner (xkblas_b200/autotune.py) in its quick mode: it measures
on the device, writes a tuning table the runtime can load, and its choices
are in range.  The moduli choice must not be worse than the plain FP64
kernel on the exponent-spread inputs it was measured on.  Requires a B200."""
import pytest

pytestmark = pytest.mark.gpu


def test_quick_autotune_writes_a_loadable_table(xk, tmp_path):
    from xkblas_b200 import autotune
    lib = xk.lib()
    table = autotune.Tuner(quick=True, log=lambda *a: None).run()
    out = tmp_path / "tune.txt"
    autotune.write_table(table, str(out))
    lib.xkb_tune_clear()
    assert lib.xkb_tune_load(str(out).encode()) == len(table)
    for k, (v, _) in table.items():
        assert lib.xkb_tune_get(k.encode(), -1.0) == float(v), k
    assert lib.xkb_tune_get(b"batch_schedule", -1) in (0.0, 1.0)
    for k, (v, note) in table.items():
        if k.startswith("ozaki_moduli_k<="):
            assert 10 <= v <= 16, (k, v)
            assert lib.xkb_ozaki_default_moduli(int(k.split("<=")[1])) == v
    lib.xkb_tune_clear()
