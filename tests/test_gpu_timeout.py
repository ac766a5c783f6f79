"""The bounded-wait path of the tensor-core evaluation kernels, made to give up on purpose.

Every mbarrier wait in EvalTcKernel and EvalTctKernel polls at most the runtime's wait limit. With the limit at 0
a wait gives up at the first phase that has not completed yet (a bulk copy or an MMA just issued), so an
evaluation takes the failure path: the CTA stops issuing copies and MMAs, waits (bounded) for the copies and MMAs
already in flight, releases its tensor memory and records NWG_TIMEOUT (17), the first-failure status convention
of the reference (slab_runtime.cu:288-290). The runtime must stay usable: the next evaluation at the default limit
gives the plain form's fitness bits (the exact forms) or the form's own earlier fitness (the trunk form).
Nothing here faults or hangs a GPU: every wait, including the wind-down's, is bounded.
"""
import numpy as np
import pytest

from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
NWG_TIMEOUT = 17


@pytest.mark.parametrize("form", [2, 4], ids=["tc-fp16-scoring", "tc-trunk-fp16"])
def test_a_wait_that_gives_up_returns_timeout_and_leaves_the_runtime_usable(form):
    action_count, population, columns, per_cell = 300, 16, 4, 9
    rng = np.random.default_rng(1717 + form)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=99)
    offsets = np.arange(population + 1, dtype=np.uint32) * per_cell
    rt.set_cell_words(offsets, np.concatenate([rng.choice(action_count, per_cell, replace=False)
                                               for _ in range(population)]).astype(np.uint32))
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    rt.evaluate(counts)
    plain = rt.current_generation()["fitness"].copy()
    rt.set_form(form)
    rt.set_margin_guard(1e-3)
    rt.evaluate(counts)
    before = rt.current_generation()["fitness"].copy()
    if form == 2:
        assert np.array_equal(before.view(np.uint32), plain.view(np.uint32))
    for attempt in range(2):  # twice in a row: the wind-down leaves nothing behind
        rt.set_wait_limit(0)
        with pytest.raises(G.nwg.NwgError) as err:
            rt.evaluate(counts)
        assert err.value.status == NWG_TIMEOUT, f"attempt {attempt}"
        rt.set_wait_limit(rt.DEFAULT_WAIT_LIMIT)
        rt.evaluate(counts)
        after = rt.current_generation()["fitness"]
        assert rt.status() == 0
        assert np.array_equal(after.view(np.uint32), before.view(np.uint32)), f"attempt {attempt}"
    rt.close()
