"""Host-only output helpers (no GPU): PRINT_STAT's formatted line and the
binary checkpoint's file layout."""
import os

import numpy as np
import pytest

from simox_b200 import _abi, checkpoint, systems as S


@pytest.fixture(scope="module")
def api_mod(simox_lib):
    from simox_b200 import api
    return api


def _fortran_es(x, w=11, d=4):
    """ES11.4 as gfortran writes it (|exponent| < 100)."""
    return f"{x:{w}.{d}E}"


def test_format_status_matches_print_stat(api_mod):
    """util.f90:3-19: time = Nloop TFM dt, T = mv2/(3N)/kB, E_es, E_eam,
    E_total = E_es + E_eam + mv2/2, FORMAT (ES11.4, 1X, F6.1, 5(1X, ES11.4))."""
    e = {"Eself": -696421.6259733407, "Edir": -1751398.1476689952, "Erec": 2523.270418048911,
         "Epair": -352348.937272716, "Egroup": -213545.07777913337, "Ectip": 302134.8784621904,
         "mv2": 32258.602966165065}
    n, step, dt = 128000, 250, 1.0 / S.TFM
    line = api_mod.format_status(e, n, step, dt)
    E_es = e["Eself"] + e["Edir"] + e["Erec"] + e["Ectip"]
    E_eam = e["Epair"] + e["Egroup"]
    E_total = E_es + E_eam + e["mv2"] / 2.0
    T = e["mv2"] / (n * 3) / 8.617343e-5
    expect = " ".join([_fortran_es(step * S.TFM * dt), f"{T:6.1f}", _fortran_es(E_total), _fortran_es(E_es),
                       _fortran_es(E_eam), _fortran_es(e["Epair"]), _fortran_es(e["Egroup"])])
    assert line == expect
    assert line == " 2.5000E+02  974.9 -2.6929E+06 -2.1432E+06 -5.6589E+05 -3.5235E+05 -2.1355E+05"


def test_format_status_overflow_and_arguments(api_mod):
    hot = {"mv2": 1e9}
    assert api_mod.format_status(hot, 10, 1, 0.1).split()[1] == "******"     # F6.1 overflow
    with pytest.raises(api_mod.SimoxError):
        api_mod.format_status(hot, 0, 1, 0.1)


def test_checkpoint_file_round_trip(tmp_path):
    s = S.small_alo(seed=5, n=300)
    rng = np.random.default_rng(2)
    v, f = rng.normal(size=(s.n, 3)), rng.normal(size=(s.n, 3))
    p = os.fspath(tmp_path / "state.ck")
    checkpoint.write(p, s.ids, s.x, v, f, s.q, s.box, step=1234567890123)
    d = checkpoint.read(p)
    assert d["n"] == s.n and d["step"] == 1234567890123
    assert np.array_equal(d["ids"], s.ids) and np.array_equal(d["box"], s.box)
    for k, a in (("x", s.x), ("v", v), ("f", f), ("q", s.q)):
        assert np.array_equal(d[k], a)
    assert os.path.getsize(p) == 48 + 4 * s.n + 80 * s.n
    with open(p, "r+b") as fh:                  # a foreign or truncated file is refused
        fh.write(b"NOTACKPT")
    with pytest.raises(ValueError):
        checkpoint.read(p)


@pytest.mark.parametrize("cut", [1, 5, 8, 47])
def test_checkpoint_truncated_by_a_few_bytes_is_refused(tmp_path, cut):
    """A file missing its last bytes fails the explicit length check with a
    clear message, not later inside numpy."""
    s = S.small_alo(seed=6, n=40)
    p = os.fspath(tmp_path / "state.ck")
    checkpoint.write(p, s.ids, s.x, s.x, s.x, s.q, s.box, step=3)
    with open(p, "rb") as fh:
        data = fh.read()
    with open(p, "wb") as fh:
        fh.write(data[:-cut])
    with pytest.raises(ValueError, match="short file"):
        checkpoint.read(p)
    with open(p, "wb") as fh:          # a bare header shorter than 48 bytes
        fh.write(data[:44])
    with pytest.raises(ValueError, match="not a checkpoint"):
        checkpoint.read(p)
