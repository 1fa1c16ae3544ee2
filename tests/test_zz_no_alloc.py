"""The allocation-free FP64 residual entry point against the regular one.

tb_residual_f64_device_static serves callers that may not allocate device
memory while they run: programs whose device memory is owned by another
allocator, and loops where cudaMalloc's implicit synchronisation would stall
them.  Its reduction scratch is a static device array instead of memory the
system allocates.  Over two calls in a row with different inputs it must give
exactly the residual b - A x of tb_apply_f64_device, the norms of that
residual, and leave the device's free memory unchanged.  The file sorts last,
so a run that stops at the first failure has run every other test first.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _board(slabs, rows, cols, seed):
    rng = np.random.default_rng(seed)
    k_in = np.where(rng.random((slabs, rows, cols)) < 0.5, 385.0, 0.3)
    robin = np.zeros((slabs + 1, rows + 1, cols + 1))
    robin[-1] = rng.uniform(0.0, 1e-5, robin[-1].shape)
    free = np.ones((slabs + 1, rows + 1, cols + 1), dtype=np.uint8)
    free[0][rng.random(free[0].shape) < 0.1] = 0
    return dict(slab_thickness_m=rng.uniform(0.03e-3, 0.5e-3, slabs), pitch_x_m=rng.uniform(0.1e-3, 0.4e-3, cols),
                pitch_y_m=rng.uniform(0.1e-3, 0.4e-3, rows), k_in=k_in, k_z=0.7 * k_in,
                robin_total=robin.reshape(-1), free_nodes=free.reshape(-1))


@pytest.mark.parametrize("shape", [(3, 31, 121), (6, 70, 45)])
def test_static_residual_matches_the_regular_entry_point_on_consecutive_calls(shape) -> None:
    import torch

    from pcb_analysis_b200._native import DeviceSystem

    dev = DeviceSystem(**_board(*shape, seed=sum(shape)))
    try:
        rng = np.random.default_rng(3)
        xs = [torch.as_tensor(rng.standard_normal(dev.size), device="cuda") for _ in range(2)]
        bs = [torch.as_tensor(rng.standard_normal(dev.size), device="cuda") for _ in range(2)]
        y, r, diff = (torch.empty_like(xs[0]) for _ in range(3))

        def both(x, b):
            r.fill_(float("nan"))
            norms = dev.residual_f64_device_static(x, b, r)
            dev.apply_f64_device(x, y)
            torch.sub(b, y, out=diff)
            return norms, r.cpu().numpy(), diff.cpu().numpy()

        # One round first: the first call on the device looks the scratch up,
        # and every kernel used here (torch's too) is loaded on first use.
        both(xs[1], bs[1])
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        for x, b in zip(xs, bs):
            (res2, peak), got, expected = both(x, b)
            np.testing.assert_array_equal(got, expected)
            assert res2 == pytest.approx(float(np.dot(expected, expected)), rel=1e-12)
            assert peak == float(np.abs(expected).max())
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before
    finally:
        dev.close()


def test_static_residual_refuses_a_board_beyond_its_scratch() -> None:
    """8192 tiles of 60 x 15 nodes; a 1 x 10000 x 1000 board needs 17 x 667."""

    import torch

    from pcb_analysis_b200._native import DeviceSystem

    dev = DeviceSystem(**_board(1, 10000, 1000, seed=1))
    try:
        dev.tile_rows = 16
        x = torch.zeros(dev.size, dtype=torch.float64, device="cuda")
        with pytest.raises(ValueError, match="static scratch"):
            dev.residual_f64_device_static(x, x, x.clone())
    finally:
        dev.close()
