"""GPU test of the chunk queue (simple3.0_b200/batching.py): chunks of the three
batching geometries, of uneven sizes, run through two worker streams must give per
chunk exactly the result of searching that chunk alone (BF16-split search with the
FP32 re-score of the top 8)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_queue_results_equal_each_chunk_alone(pkg):
    b = pkg.batching
    spec = [("A", 14, 70), ("B", 9, 33), ("C", 5, 21), ("A", 23, 48), ("B", 6, 57), ("C", 7, 12)]
    chunks = [b.synthetic_chunk(g, nr, npt, seed=i) for i, (g, nr, npt) in enumerate(spec)]
    got = b.SearchQueue(workers=2).run(chunks)
    for ch, res in zip(chunks, got):
        alone = b.search_chunk(ch)
        assert res.shape == (ch.nptcls,)
        for f in ("iref", "irot", "ishift"):
            assert np.array_equal(res[f], alone[f])
        assert np.array_equal(res["corr"].view(np.int32), alone["corr"].view(np.int32))
        assert np.all(res["iref"] >= 1) and np.all(res["iref"] <= ch.nrefs)
