"""bench.py's command line: the default step counts per workload and the
reference arm (host only; no GPU call)."""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _parse(argv, monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"] + argv)
    return _bench().parse()


def test_default_steps_per_workload(monkeypatch):
    assert _parse([], monkeypatch).steps == 100  # the 3-D explosion's run length
    assert _parse(["--workload", "amr"], monkeypatch).steps == 20
    for w in ("batch", "adjoint", "batch_adjoint"):
        assert _parse(["--workload", w], monkeypatch).steps == 3
    assert _parse(["--impl", "reference"], monkeypatch).steps == 3


def test_driver_flags_override_the_defaults(monkeypatch):
    a = _parse(["--gpus", "4", "--steps", "7", "--warmup", "5"], monkeypatch)
    assert (a.gpus, a.steps, a.warmup, a.impl, a.workload) == (4, 7, 5, "ours", "uniform")
    assert _parse([], monkeypatch).warmup >= 3  # at least 3 untimed warm-up steps


def test_reference_gpu_leg_is_on_by_default(monkeypatch):
    assert _parse([], monkeypatch).reference_gpu is True
    assert _parse(["--no-reference-gpu"], monkeypatch).reference_gpu is False


def test_fast_form_is_a_uniform_workload_option(monkeypatch):
    import pytest
    assert _parse(["--precision", "fast"], monkeypatch).precision == "fast"
    with pytest.raises(SystemExit):
        _parse(["--precision", "fast", "--workload", "adjoint"], monkeypatch)


def test_subrecords_are_on_by_default(monkeypatch):
    assert _parse([], monkeypatch).no_subrecords is False
    assert _parse(["--no-subrecords"], monkeypatch).no_subrecords is True


def test_reference_gpu_leg_reports_a_missing_library(monkeypatch, tmp_path):
    """Without oracle/_ref/librefgpu.so the leg says so instead of failing
    (it returns before any device call)."""
    bench = _bench()
    from oracle import pyrefgpu
    monkeypatch.setattr(pyrefgpu, "LIB_PATH", str(tmp_path / "librefgpu.so"))
    out = bench.reference_gpu_leg(None, None, None, None, None, 0, 1.0, None)
    assert "unavailable" in out and "librefgpu.so" in out["unavailable"]
