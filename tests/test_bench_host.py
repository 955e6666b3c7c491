"""Host logic of bench.py (no GPU): which form a line reports."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def forms(**kw):
    base = {"plain_fp64": {"t": 3.6, "bwd": 3e-19, "inertia": (216000, 54000, 0)}}
    base.update(kw)
    return base


def test_fastest_accurate_form_is_chosen():
    f = forms(mixed={"t": 0.65, "bwd": 2e-15, "inertia": (216000, 54000, 0)},
              tf32={"t": 0.9, "bwd": 1e-15, "inertia": (216000, 54000, 0)})
    assert bench.choose_form(f) == "mixed"


def test_inaccurate_or_wrong_inertia_forms_are_not_chosen():
    f = forms(slow_ok={"t": 1.2, "bwd": 1e-15, "inertia": (216000, 54000, 0)},
              inaccurate={"t": 0.5, "bwd": 3e-6, "inertia": (216000, 54000, 0)},
              flipped={"t": 0.4, "bwd": 4e-15, "inertia": (216001, 53999, 0)})
    assert bench.choose_form(f) == "slow_ok"


def test_plain_form_always_qualifies():
    f = forms(flipped={"t": 0.4, "bwd": 4e-15, "inertia": (950001, 49999, 0)})
    assert bench.choose_form(f) == "plain_fp64"


def test_form_dtype_names_the_arithmetic():
    import importlib
    rv = importlib.import_module("__graft_entry__").load_package()
    assert bench.form_dtype(rv.FactorOptions(precision="fp64")) == "f64"
    assert bench.form_dtype(rv.FactorOptions(precision="mixed", mixed_operands="bf16")).startswith("bf16x3")
    assert bench.form_dtype(rv.FactorOptions(precision="learned", mixed_operands="bf16")).startswith("learned")
