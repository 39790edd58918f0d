"""The batched path's autotuner (psm_autotune_batch) and its settings.

The tuner times a sample batch under every candidate setting (preparation
team, initial work pieces per enumeration warp, enumeration grid, then the
intersection variant), keeps the fastest and installs it in the context.
Settings change how the work is spread over the GPU, never the counts.
"""
import ctypes as C

import pytest

from psm_benchmark_b200 import api, gen
from psm_benchmark_b200 import native as N
from psm_benchmark_b200.native import PsmError
from tests import golden_data as gd

pytestmark = pytest.mark.gpu


def test_autotune_keeps_counts_and_installs_the_fastest_setting():
    g = gd.synthetic_graph("rmat12")
    queries = gen.make_queries(g, [4, 6, 8, 12] * 10, gen.BASE_SEED + 91)
    with api.Engine(arena_bytes=2 << 30) as eng:
        dg = api.DataGraph.from_graph(g)
        assert eng.batch_tuning() == {"team": "RULE", "grabs_per_warp": 8, "enum_quarters": 4, "intersect": "BINARY",
                                      "ms": 0.0}
        before = [r.count for r in api.match_batch(eng, dg, queries, "CFL_CFL_EXPLORE", cap=10**5)]
        t = eng.autotune_batch(dg, queries, "CFL_CFL_EXPLORE", cap=10**5, repeats=1)
        tried = t["tried"]
        assert len(tried) >= 6
        # the intersection variants are tried under the best of the others
        assert {x["intersect"] for x in tried} == {"AUTO", "BINARY", "MERGE"}
        assert t["best"]["ms"] == min(x["ms"] for x in tried)
        assert t["best"] in tried
        installed = eng.batch_tuning()
        for k in ("team", "grabs_per_warp", "enum_quarters", "intersect"):
            assert installed[k] == t["best"][k]
        # every setting counts the same embeddings
        for x in tried:
            eng.set_batch_tuning(x["team"], x["grabs_per_warp"], x["enum_quarters"], x["intersect"])
            assert [r.count for r in api.match_batch(eng, dg, queries, "CFL_CFL_EXPLORE", cap=10**5)] == before
        dg.close()


def test_batch_tuning_rejects_out_of_range_settings():
    with api.Engine(arena_bytes=1 << 30) as eng:
        for bad in (dict(grabs_per_warp=0), dict(grabs_per_warp=65), dict(enum_quarters=0), dict(enum_quarters=5)):
            with pytest.raises(PsmError):
                eng.set_batch_tuning(**bad)
        t = N.BatchTuning(1, 8, 4, 3, 0.0)  # no fourth intersection variant
        with pytest.raises(PsmError):
            N.check(N.lib().psm_context_set_batch_tuning(eng._h, C.byref(t)))
        eng.set_batch_tuning("BLOCK", 2, 2)
        assert eng.batch_tuning()["team"] == "BLOCK"
