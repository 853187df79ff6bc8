"""The autotuner's choice and cache logic (no GPU: a fake timer stands in for the device)."""
from __future__ import annotations

import json
from types import SimpleNamespace

import pytest


def _mod(f3d):
    import importlib
    return importlib.import_module(f3d.__name__ + ".autotune")


def _dc(ns=3, cells=64 ** 3, precision=1):
    return SimpleNamespace(precision=precision, case=SimpleNamespace(ns=ns, cells=cells))


def test_picks_fastest_and_caches(f3d, tmp_path):
    A = _mod(f3d)
    calls = []
    times = {0: 5.0, 1: 4.0, 2: 6.0, 3: 2.5, 4: 2.0, 5: 2.2, 6: 2.1}

    def measure(dc, tile):
        calls.append(tile)
        return times[tile]

    t = A.Autotuner(tmp_path / "a.json", measure=measure)
    assert t.choose(_dc(), gpu="B200") == 4
    assert sorted(calls) == list(A.CANDIDATES)
    assert t.choose(_dc(), gpu="B200") == 4 and len(calls) == len(A.CANDIDATES)  # cached
    saved = json.loads((tmp_path / "a.json").read_text())
    k = A.key("B200", 1, 3, 64 ** 3)
    assert saved[k]["tile"] == 4 and set(saved[k]["ms_per_step"]) == {str(t) for t in A.CANDIDATES}
    t2 = A.Autotuner(tmp_path / "a.json", measure=lambda dc, tile: pytest.fail("re-timed"))
    assert t2.choose(_dc(), gpu="B200") == 4  # read back from the file


def test_keys_separate_precision_species_and_size(f3d, tmp_path):
    A = _mod(f3d)
    seen = []
    t = A.Autotuner(tmp_path / "b.json", measure=lambda dc, tile: seen.append(tile) or tile)
    t.choose(_dc(ns=1), gpu="g")
    t.choose(_dc(ns=2), gpu="g")
    t.choose(_dc(ns=2, precision=0), gpu="g")
    t.choose(_dc(ns=2, cells=128 ** 3), gpu="g")
    t.choose(_dc(ns=2, cells=64 ** 3 + 1000), gpu="g")  # same size class: cached
    assert len(seen) == 4 * len(A.CANDIDATES)
    assert A.size_class(64 ** 3) == 18 and A.size_class(128 ** 3) == 21


def test_failing_configuration_is_skipped(f3d, tmp_path):
    A = _mod(f3d)

    def measure(dc, tile):
        if tile == 3:
            raise RuntimeError("does not fit")
        return {0: 3.0, 1: 2.0, 2: 9.0, 4: 5.0, 5: 6.0, 6: 7.0}[tile]

    t = A.Autotuner(tmp_path / "c.json", measure=measure)
    assert t.choose(_dc(), gpu="g") == 1


def test_unwritable_cache_still_chooses(f3d, tmp_path):
    A = _mod(f3d)
    blocker = tmp_path / "file"
    blocker.write_text("x")
    t = A.Autotuner(blocker / "sub" / "d.json", measure=lambda dc, tile: 10 - tile)
    assert t.choose(_dc(), gpu="g") == max(A.CANDIDATES)
