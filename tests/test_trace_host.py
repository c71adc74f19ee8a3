"""Phase tracing (edrixs_b200.trace) on the host: off by default, records and prints when on."""
import pytest

from edrixs_b200 import trace


@pytest.fixture
def tracing():
    level = trace._level
    trace.records.clear()
    yield trace
    trace.enable(level)
    trace.records.clear()


def test_disabled_phase_records_nothing(tracing):
    tracing.enable(0)
    with tracing.phase("x"):
        pass
    assert tracing.records == [] and not tracing.enabled()


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="host-only path (no CUDA events)")
def test_enabled_phases_record_nest_and_survive_errors(tracing, capsys):
    tracing.enable(2)
    with tracing.phase("outer"):
        with tracing.phase("inner"):
            pass
    with pytest.raises(ValueError):
        with tracing.phase("inner"):
            raise ValueError("boom")
    names = [r["phase"] for r in tracing.records]
    assert names == ["inner", "outer", "inner"]
    assert [r["ok"] for r in tracing.records] == [True, True, False]
    assert all(r["wall_ms"] >= 0 and r["device_ms"] is None for r in tracing.records)
    s = tracing.summary()
    assert s["inner"]["calls"] == 2 and s["outer"]["calls"] == 1
    out = capsys.readouterr().out.splitlines()
    assert len(out) == 3 and out[0].startswith("edx >>> inner: wall ")
