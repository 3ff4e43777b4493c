"""GIZMO built with the B200 gravity path has no CPU fallback.

On a host without a CUDA device the library's gg_create reports
GG_ERR_CUDA, and the host code (gizmo-public_b200/host/gravtree_b200.c)
turns any nonzero status into GIZMO's endrun(): the run stops with the
library's message instead of computing gravity some other way.
"""
import pytest

import ics
import ref_runner


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a CUDA device is present: the GIZMO integration test runs the real path")
@pytest.mark.skipif(not ref_runner.available(ref_runner.BIN_B200),
                    reason="GIZMO+B200 binary not built (oracle/build_ref.sh needs the reference tree)")
def test_gizmo_with_b200_gravity_stops_without_a_device():
    ic = ics.plummer(300, seed=5)
    with pytest.raises(RuntimeError) as e:
        ref_runner.run(ic, tol=0.0025, threads=1, binary=ref_runner.BIN_B200)
    msg = str(e.value)
    assert "gg_create failed" in msg and "no CUDA device" in msg and "ENDRUN" in msg
