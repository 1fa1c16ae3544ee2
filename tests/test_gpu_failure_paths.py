"""The give-up path of the operator's tensor-copy staging, without a GPU fault.

Every wait of the FP32 operator on its staged tiles is bounded; a block that
gives up votes the timeout through the block, lets its copies in flight land,
sets the system's error word and the solve state, and returns.  Here the
test switch (tb_set_stage_test) arms the stage barriers without issuing any
copy, so the waits run out with nothing in flight.  Checked: the apply and
the MPIR solve fail with TimeoutError (TB_ETIMEOUT), not a wrong status, and
once the switch is off the same system gives the same bits as before.
"""

from __future__ import annotations

import numpy as np
import pytest

from pcb_analysis_b200._native import DeviceSystem
from pcb_analysis_b200.mpir import MPIRConfig

pytestmark = pytest.mark.gpu

CONFIG = MPIRConfig(inner_relative_tolerance=1e-4, max_outer_iterations=30, max_inner_iterations=100000)


def _arrays(slabs=4, rows=40, cols=70, seed=11):
    rng = np.random.default_rng(seed)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.5, 385.0, 0.3)
    node_shape = (slabs + 1, rows + 1, cols + 1)
    robin = np.zeros(node_shape)
    robin[-1] = 1e-6
    rhs = np.zeros(node_shape)
    rhs[-1, rows // 2, cols // 2] = 1e-2
    arrays = dict(slab_thickness_m=np.full(slabs, 0.2e-3), pitch_x_m=np.full(cols, 0.25e-3),
                  pitch_y_m=np.full(rows, 0.25e-3), k_in=k_in, k_z=k_in, robin_total=robin.reshape(-1),
                  free_nodes=np.ones(int(np.prod(node_shape)), dtype=np.uint8))
    return arrays, rhs.reshape(-1)


@pytest.mark.parametrize("plan", [(0, 16, 1, 0, 0), (2, 8, 1, 0, 0)])
def test_a_stage_wait_that_runs_out_is_reported_and_the_system_stays_usable(plan) -> None:
    arrays, rhs = _arrays()
    with DeviceSystem(**arrays) as dev:
        dev.apply_plan = plan
        x = np.random.default_rng(1).standard_normal(dev.size).astype(np.float32)
        before = dev.apply_f32(x)
        solved = dev.solve_mpir(rhs, CONFIG)
        assert solved["converged"]
        dev.set_stage_test(64)
        with pytest.raises(TimeoutError, match="staged tiles"):
            dev.apply_f32(x)
        with pytest.raises(TimeoutError):
            dev.solve_mpir(rhs, CONFIG)
        dev.set_stage_test(0)
        np.testing.assert_array_equal(dev.apply_f32(x), before)
        again = dev.solve_mpir(rhs, CONFIG)
        np.testing.assert_array_equal(again["solution"], solved["solution"])
        assert again["history"] == solved["history"]
