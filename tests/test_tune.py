"""The autotuner's bookkeeping on the CPU (efmm_tune_*): exploration order,
the decision after every candidate's timed runs, per-key separation, and
persistence of decisions through ELFMM3D_TUNE_FILE."""
import ctypes

import elfmmlib3d_b200 as E


def _L():
    L = E.load()
    L.efmm_tune_pick.restype = ctypes.c_int
    L.efmm_tune_pick.argtypes = [ctypes.c_int] * 7
    L.efmm_tune_report.restype = None
    L.efmm_tune_report.argtypes = [ctypes.c_int] * 8 + [ctypes.c_float]
    return L


KEY = (1, 30, 480, 256, 1, 0)  # knob (M2L), order, leaf capacity, columns, precision, plan kind


def _explore(L, key, times):
    """Run the tuner's protocol: pick, 'run' (report the given time)."""
    picks = []
    for _ in range(2 * len(times)):
        c = L.efmm_tune_pick(*key, len(times))
        picks.append(c)
        L.efmm_tune_report(*key, len(times), c, times[c])
    return picks


def test_explores_each_candidate_then_keeps_the_fastest(monkeypatch):
    monkeypatch.delenv("ELFMM3D_TUNE_FILE", raising=False)
    L = _L()
    L.efmm_tune_reset()
    assert _explore(L, KEY, [5.0, 3.0]) == [0, 0, 1, 1]
    assert L.efmm_tune_pick(*KEY, 2) == 1
    assert L.efmm_tune_pick(*KEY, 2) == 1
    # another key (other columns) is explored on its own
    other = KEY[:3] + (64,) + KEY[4:]
    assert L.efmm_tune_pick(*other, 2) == 0
    lines = E.tune_dump()
    assert any(l.startswith("1 30 480 256 1 0 1 5.0000 3.0000") for l in lines)
    L.efmm_tune_reset()
    assert E.tune_dump() == []


def test_decisions_persist_in_the_tune_file(tmp_path, monkeypatch):
    f = tmp_path / "tune.txt"
    monkeypatch.setenv("ELFMM3D_TUNE_FILE", str(f))
    L = _L()
    L.efmm_tune_reset()
    _explore(L, KEY, [2.0, 4.0])
    assert L.efmm_tune_pick(*KEY, 2) == 0
    assert f.read_text().split()[:7] == ["1", "30", "480", "256", "1", "0", "0"]
    L.efmm_tune_reset()  # a later process: the decision is read back, no exploration
    assert L.efmm_tune_pick(*KEY, 2) == 0
    L.efmm_tune_reset()
    monkeypatch.delenv("ELFMM3D_TUNE_FILE")
    L.efmm_tune_reset()
