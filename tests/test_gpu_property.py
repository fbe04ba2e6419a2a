"""Property test of the CUDA path against the oracle on adversarial small inputs:
duplicates, lattice points exactly eps apart, NaN, inf, FLT_MAX (the reference's
padding marker in coordinate 0), subnormals, eps of 0 or negative, minPts from 0
to past n, every d from 1 to 16.  Counts, ids and meta must be bit-identical, in
both count modes and through the batched entry point."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_gpu_matches_oracle_on_adversarial_inputs(ctx):
    hyp = pytest.importorskip("hypothesis")
    st = pytest.importorskip("hypothesis.strategies")
    fmax = float(np.finfo(np.float32).max)
    values = st.sampled_from([0.0, 0.25, 0.5, 0.75, 1.0, -0.5, 3.0, 1e-40, float("nan"), float("inf"),
                              -float("inf"), fmax, 0.1, 0.2, 0.3])
    seen = []

    @hyp.settings(max_examples=120, deadline=None, derandomize=True,
                  phases=[hyp.Phase.explicit, hyp.Phase.generate])
    @hyp.given(d=st.integers(1, 16), n=st.integers(1, 40), data=st.data(),
               eps=st.sampled_from([0.0, 0.25, 0.5, -0.5, 0.3, 1.0, 2.5]), m=st.integers(0, 8))
    def check(d, n, data, eps, m):
        flat = data.draw(st.lists(values, min_size=n * d, max_size=n * d))
        x = np.array(flat, dtype=np.float32).reshape(n, d)
        nn_o, ci_o, _, meta = oracle.reference(x, eps, m)
        nn, ci, res = ctx.run(x, eps, m, full_count=True)
        np.testing.assert_array_equal(nn, nn_o)
        np.testing.assert_array_equal(ci, ci_o)
        assert (res.clusters, res.noise, res.core_count) == (meta["clusters"], meta["noise"], meta["cores"])
        _, ci_e, _ = ctx.run(x, eps, m)
        np.testing.assert_array_equal(ci_e, ci_o)
        seen.append((x, eps, m, ci_o))

    check()
    # the same problems as one batch
    outs = ctx.run_batched([(x, e, m) for x, e, m, _ in seen])
    for (x, e, m, ci_o), (_, ci, _) in zip(seen, outs):
        np.testing.assert_array_equal(ci, ci_o)
