"""The serving form (openhomelbm_b200.serving) on the GPU: a request's per-segment loads are
the same whether it runs alone or in a mix of concurrently stepped domains, the served
pipeline (one CUDA graph per control step, poses through the coupling kernel) computes what
the plain solver computes, and admission respects the slot count and the HBM budget.

Loads are compared to 1e-6 of the largest load magnitude: the per-solid sums are binary64
atomics whose order varies between runs; every other value is computed identically.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _close(a, b, tol=1e-6):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return a.shape == b.shape and np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-30)


def _reqs():
    from openhomelbm_b200.serving import Request

    return [Request(0, 64, 11, 0.0, control_steps=3, substeps=4), Request(1, 96, 12, 0.0, control_steps=4, substeps=4),
            Request(2, 64, 13, 0.0, control_steps=2, substeps=4)]


def test_result_alone_equals_result_in_mix():
    from openhomelbm_b200.serving import ServeEngine

    reqs = _reqs()
    alone = ServeEngine(storage="float16", max_active=1).run([reqs[0]], realtime=False)
    mix = ServeEngine(storage="float16", max_active=3).run(reqs, realtime=False)
    assert mix.max_active == 3
    assert set(mix.results) == {0, 1, 2}
    assert alone.results[0].shape == (3, 4, 5, 6)
    assert np.abs(alone.results[0]).max() > 0
    assert _close(mix.results[0], alone.results[0])
    assert mix.env_steps == 3 + 4 + 2


def test_served_pipeline_matches_plain_solver():
    from openhomelbm_b200.serving import ServeEngine, run_plain

    reqs = _reqs()
    served = ServeEngine(storage="float32", max_active=3).run(reqs, realtime=False)
    plain = run_plain(reqs, storage="float32")
    for r in reqs:
        assert _close(served.results[r.rid], plain.results[r.rid], 1e-5), r.rid


def test_admission_respects_slots_and_budget():
    from openhomelbm_b200.serving import ServeEngine, domain_bytes

    reqs = _reqs()
    one_slot = ServeEngine(storage="float16", max_active=2).run(reqs, realtime=False)
    assert one_slot.max_active == 2
    budget = domain_bytes(96, "float16") + domain_bytes(64, "float16") // 2
    tight = ServeEngine(storage="float16", max_active=8, budget_bytes=budget).run(reqs, realtime=False)
    assert tight.max_active == 1
    assert set(tight.results) == {0, 1, 2}


@pytest.mark.parametrize("batched", [False, True])
def test_x_split_of_served_domains_does_not_change_results(batched):
    """ServeEngine(x_chunks=k, link_blocks=b) runs its domains' stream-collide with k x chunks
    per tile column and their cut links on b blocks (0: the library's automatic choices) and
    restores the process-wide settings afterwards; the split and the grid change which CTA
    computes a plane or a cell, not what it computes."""
    from openhomelbm_b200 import _lib
    from openhomelbm_b200.serving import ServeEngine

    reqs = _reqs()
    _lib.set_tuning("d3q27_chunks", 0)
    _lib.set_tuning("d3q27_link_blocks", 0)
    blocks = {0: 0, 1: 148, 3: 37}  # the cut-link grid changes which block takes a cell, too
    runs = {k: ServeEngine(storage="float16", max_active=3, batched=batched, x_chunks=k, link_blocks=blocks[k],
                           keep_fields=True).run(reqs, realtime=False) for k in (0, 1, 3)}
    assert _lib.get_tuning("d3q27_chunks") == 0 and _lib.get_tuning("d3q27_link_blocks") == 0
    for k in (1, 3):
        for r in reqs:
            np.testing.assert_array_equal(runs[k].fields[r.rid], runs[0].fields[r.rid])
            assert _close(runs[k].results[r.rid], runs[0].results[r.rid])
    with pytest.raises(ValueError):
        ServeEngine(x_chunks=-1)
    with pytest.raises(ValueError):
        ServeEngine(link_blocks=-1)
