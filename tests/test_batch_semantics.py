"""The batched integrands' default semantics (a fixed budget of ncalls drawn
points per multichannel task, option batch_retry 0) against the reference's
retry loop (MultiChannel.hh:214-248, option batch_retry 1), on the C oracle
(pinned to the compiled reference by tests/test_oracle_pin.py).

Task 422 of the 512-integrand benchmark batch (2->4, 15 channels, 422750
calls, PreProcess = finite momenta) under the retry loop has NaN channel
weights after its third adaptation, and its fourth iteration finds no point
with a finite value: the reference's loop would not end, and the GPU's retry
mode stops with CHILI_ERR_TIMEOUT after max_rounds rounds.  Under the fixed
budget the same task stays finite.  This is why the fixed budget is the
batch's default."""
import numpy as np

from chili_b200 import workloads
from oracle import port

TASK = 422


def _oracle(t, k, fixed):
    cs = t["channels"]
    params = workloads.mc_params(t["ncalls"], beta=t["beta"], min_alpha=t["min_alpha"], grid_alpha=t["grid_alpha"])
    O = port.MultiChannel(cs, t["bins"], params, t["fkind"], t["params"], pre=t["pre"])
    O.set_fixed_budget(fixed)
    return O, cs


def test_retry_loop_turns_task_422_nan_and_fixed_budget_does_not():
    tasks = workloads.batched_tasks(seed=2024)
    t = tasks[TASK]
    assert t["kind"] == "multichannel" and t["ncalls"] == 422750
    O, cs = _oracle(t, TASK, fixed=False)
    tried = []
    for it in range(3):
        u = port.philox_uniforms(2024 + TASK, it << 32, 3 * t["ncalls"], cs.ndims + 1)
        st, info = O.iterate(u)
        tried.append(info.points_tried)
        assert st.n == info.points_tried
    assert tried == [1099338, 661702, 550047]
    assert np.isnan(O.get_alpha()[0]).all()
    F, _ = _oracle(t, TASK, fixed=True)
    for it in range(3):
        u = port.philox_uniforms(2024 + TASK, it << 32, t["ncalls"], cs.ndims + 1)
        st, _ = F.iterate(u)
        assert np.isfinite(st.sum) and st.n == t["ncalls"]
    assert np.isfinite(F.get_alpha()[0]).all()
