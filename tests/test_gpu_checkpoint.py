"""Binary FP64 checkpoint (simox_checkpoint_write / _read) on the GPU.

A run restarted from a checkpoint in a fresh context continues the original
trajectory: after four more NVT steps positions agree to 1e-10 A (the FP64
PME spread sums in atomic order, so the two runs are not bitwise equal), where
a restart from the reference's restart.xyz precision (ES13.6 positions, ES11.4
velocities and forces) departs by far more.  The file's arrays equal the
state bit for bit, and a checkpoint of another box is refused."""
import os

import numpy as np
import pytest

from simox_b200 import _abi, api, checkpoint, systems as S

from tests.helpers import gpu_context

pytestmark = pytest.mark.gpu

DT = 1.0 / S.TFM
T_GIVEN = 600.0 * S.KB


def _system(box=(31.0, 32.0, 33.0)):
    return S.small_alo(seed=12, n=500, box=box, fft=(24, 24, 24), order=4)


def _lossy(a, digits):
    return np.array([float(f"{v:.{digits}E}") for v in a.ravel()]).reshape(a.shape)


def test_checkpoint_restart_continues_trajectory(tmp_path):
    s = _system()
    p = os.fspath(tmp_path / "run.ck")
    with gpu_context(s) as g:
        g.pme_self()
        g.cell_sort()
        g.force()
        g.pme()
        g.md_run(3, DT, first_step=1, thermostat=True, T_given=T_GIVEN)
        g.checkpoint_write(p, step=3)
        st = g.get_state()
        d = checkpoint.read(p)
        assert d["step"] == 3 and np.array_equal(d["box"], s.box)
        for k in ("x", "v", "f", "q"):
            assert np.array_equal(d[k], st[k]), k
        e_ref = g.md_run(4, DT, first_step=4, thermostat=True, T_given=T_GIVEN)
        ref = g.get_state()

    def restart(x, v, f, q):
        with gpu_context(s) as h:
            if x is None:
                assert h.checkpoint_read(p) == 3
            else:
                h.set_state(x=x, v=v, f=f, q=q)
            h.pme_self()
            h.cell_sort()
            e = h.md_run(4, DT, first_step=4, thermostat=True, T_given=T_GIVEN)
            return e, h.get_state()

    e, got = restart(None, None, None, None)
    dx = np.abs(got["x"] - ref["x"]).max()
    assert dx <= 1e-10
    assert np.abs(got["v"] - ref["v"]).max() <= 1e-9 * np.abs(ref["v"]).max()
    assert abs(e["mv2"] - e_ref["mv2"]) <= 1e-10 * e_ref["mv2"]
    # the same restart at restart.xyz precision
    _, lossy = restart(_lossy(st["x"], 6), _lossy(st["v"], 4), _lossy(st["f"], 4), _lossy(st["q"], 6))
    assert np.abs(lossy["x"] - ref["x"]).max() > 100 * max(dx, 1e-14)


def test_checkpoint_of_another_box_is_refused(tmp_path):
    s = _system()
    p = os.fspath(tmp_path / "a.ck")
    with gpu_context(s) as g:
        g.checkpoint_write(p, step=1)
    with gpu_context(_system(box=(31.0, 32.0, 34.0))) as h:
        with pytest.raises(api.SimoxError) as err:
            h.checkpoint_read(p)
        assert err.value.code == _abi.SIMOX_E_IO
        with pytest.raises(api.SimoxError) as err:
            h.checkpoint_read(os.fspath(tmp_path / "missing.ck"))
        assert err.value.code == _abi.SIMOX_E_IO
