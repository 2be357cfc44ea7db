"""The super-tile autotuner: every candidate it picks is a legal side for the mesh, the choice
is cached per GPU and build, and an ensemble built with the tuned sides steps to the same
bits as with the default side (the side changes the work split, never the result)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_picks_legal_tiles_and_caches(tmp_path, monkeypatch):
    from pbh_b200 import tune
    monkeypatch.setattr(tune, "CACHE", tmp_path / "cache.json")
    got = tune.autotune([16, 32], steps=3, warmup=1)
    assert set(got) == {16, 32}
    for N, t in got.items():
        assert t in tune.CANDIDATES and t <= N
        assert set(tune.tuned_times(N)) == {str(c) for c in tune.CANDIDATES if c <= N}
    assert (tmp_path / "cache.json").exists()
    assert tune.autotune([16, 32]) == got                 # served from the cache


def test_tile_side_does_not_change_results():
    from pbh_b200 import recipe
    from pbh_b200.batch import Ensemble
    specs = [recipe.single_peak(N=32, steps=20, seed=3), recipe.single_peak(N=16, steps=20, seed=4)]
    out = []
    for tiles in ({32: 16, 16: 16}, {32: 4, 16: 8}):
        ens = Ensemble(specs, tiles=tiles)
        ens.load()
        ens.step(8)
        out.append([ens.engine.delta(i).cpu().numpy() for i in range(2)])
        ens.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
