"""Failure detection of the X/Y TMA sweep's bounded tile wait, without a GPU fault.

adi_set_fault_injection(h, ADI_FAULT_SKIP_TILE_LOADS) makes the TMA-fed X/Y
sweeps issue no tile load at all, so the mbarrier their CTAs wait on never
completes and the wait gives up after its short limit (16 polls of about 10 us):
each CTA raises the handle's device flag and leaves without writing that tile,
with no copy in flight.  The step reports ADI_ERR_TIMEOUT and leaves the layers
unswapped; with the knob cleared the context is still usable and the next step
equals a solver that never saw the fault, bit for bit.
"""
import numpy as np
import pytest

from adi_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _solver(adi_lib, d, graphs):
    from adi_b200 import _abi
    s = adi_lib.AdiSolver3D(d, params=adi_lib.fluid_params_normalized(130.0, 0.72, 1.4), solver=_abi.ADI_SOLVER_FAST)
    s.CreateSegments()
    for dr, (K, NL) in enumerate([(8, -16), (4, -8), (4, 0)]):
        s.set_fast_shape(dr, K, NL)
    s.set_graphs(graphs)
    return s


@pytest.mark.parametrize("graphs", [True, False], ids=["graph", "direct"])
def test_tile_wait_timeout_is_reported_and_the_handle_recovers(adi_lib, graphs):
    from adi_b200 import _abi
    d = G.random_domain(64, 32, 32, seed=81, shell=True, n_obstacles=8, rmax=4.5)
    s = _solver(adi_lib, d, graphs)
    ref = _solver(adi_lib, d, graphs)
    start = s.fields(0)

    s.set_fault_injection(_abi.ADI_FAULT_SKIP_TILE_LOADS)
    assert s.step(8e-4, 2, 2, True) == _abi.ADI_ERR_TIMEOUT
    msg = s.lib.adi_last_error_string(s.h).decode()
    assert "wait" in msg, msg
    for f0, f1 in zip(start, s.fields(0)):
        assert np.array_equal(f0, f1)          # layers left unswapped

    s.set_fault_injection(_abi.ADI_FAULT_NONE)
    for _ in range(2):
        assert s.step(8e-4, 2, 2, True) == 0
        assert ref.step(8e-4, 2, 2, True) == 0
    for a, b in zip(s.fields(0), ref.fields(0)):
        assert np.array_equal(a, b)
    assert s.div_error() == ref.div_error()


def test_fault_injection_rejects_unknown_modes(adi_lib):
    from adi_b200 import _abi
    d = G.random_domain(24, 20, 16, seed=3)
    s = adi_lib.AdiSolver3D(d)
    with pytest.raises(_abi.AdiError):
        s.set_fault_injection(7)
