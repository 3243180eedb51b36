"""Batched independent systems (simox_batch_*): one CUDA graph launch per MD
step for all members must give each member the trajectory it has when it is
stepped alone, and the force pass's CTA split (the autotuner's knob) must not
change any result.

Bars: FP64 positions within 1e-9 A and energies within 1e-9 relative after 8
steps (the PME spread's FP64 atomics may add in a different order); mixed
positions within 1e-6 A (batched cuFFT plans may round differently from one
system's plan); forces for CTA splits 1 and 8 bit-identical.  A mixed batch
runs in the per-pass mode (each kernel of a step launched once for all
systems); an FP64 batch, whose full-list kernels have no batched form, in the
per-system mode.
"""
import numpy as np
import pytest

from simox_b200 import api, systems as S

pytestmark = pytest.mark.gpu

DT = 1.0 / S.TFM


@pytest.fixture(scope="module", autouse=True)
def _lib(simox_lib):
    return simox_lib


def _members():
    return [S.replica(11, 700, 0.0, 300.0), S.replica(12, 1500, 0.3, 600.0),
            S.replica(13, 2600, 0.5, 900.0), S.replica(14, 4100, 0.6, 1200.0)]


def _prepared(s, precision):
    g = api.from_system(s, precision=precision)
    g.pme_self()
    g.cell_sort()
    g.force()
    g.pme()
    return g


def _opts(s):
    return api.md_opts(DT, thermostat=True, T_given=s.meta["T"] * S.KB, freq_stat=4)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_batch_matches_single_systems(precision, tol):
    systems = _members()
    alone = []
    for s in systems:
        with _prepared(s, precision) as g:
            e = g.md_run(8, DT, first_step=1, thermostat=True, T_given=s.meta["T"] * S.KB, freq_stat=4)
            alone.append((g.get_state()["x"], e))
    members = [_prepared(s, precision) for s in systems]
    try:
        with api.Batch(members) as b:
            es = b.md_run([_opts(s) for s in systems], 8, first_step=1)
            assert b.launch_count() > 0
            assert b.mode() == ("per_pass" if precision == "mixed" else "per_system")
        for k, g in enumerate(members):
            x = g.get_state()["x"]
            d = x - alone[k][0]
            d -= systems[k].box * np.round(d / systems[k].box)
            assert np.abs(d).max() <= tol, (k, np.abs(d).max())
            for key in ("Epair", "Egroup", "Edir", "Ectip", "Erec", "mv2"):
                ref = alone[k][1][key]
                assert abs(es[k][key] - ref) <= 1e-9 * max(1.0, abs(ref)) * (1 if precision == "fp64" else 1e3), key
    finally:
        for g in members:
            g.close()


def test_force_split_does_not_change_forces():
    s = S.replica(21, 3000, 0.4, 600.0)
    out = []
    for splits in (1, 8):
        with _prepared(s, "mixed") as g:
            g.set_tuning(splits)
            assert g.get_tuning()["force_splits"] == splits
            g.vv_nve1(DT)
            g.cell_sort()
            g.force(energies=False)
            out.append(g.get_state()["f"])
    assert np.array_equal(out[0], out[1])


def test_batch_autotune_picks_a_rule_and_keeps_running():
    systems = _members()
    members = [_prepared(s, "mixed") for s in systems]
    try:
        with api.Batch(members) as b:
            opts = [_opts(s) for s in systems]
            b.md_run(opts, 2, first_step=1)
            times, best = b.autotune(opts, first_step=3, trial_steps=2)
            assert np.all(times > 0) and 0 <= best < 5 and times[best] == times.min()
            e = b.md_run(opts, 4, first_step=3 + 5 * 3)
            assert all(np.isfinite(v["mv2"]) and v["mv2"] > 0 for v in e)
    finally:
        for g in members:
            g.close()


def test_batch_follows_changed_step_options():
    """A batch whose members' dt and T_given change between md_run calls
    (an annealing schedule) must step with the new values, as each context's
    own simox_md_run does -- not replay the graph captured with the old ones."""
    systems = _members()[:3]
    plan = [(DT, 1.0), (0.5 * DT, 1.6), (DT, 0.7)]     # (dt, T scale) per md_run call
    alone = []
    for s in systems:
        with _prepared(s, "fp64") as g:
            step = 1
            for dt, ts in plan:
                g.md_run(4, dt, first_step=step, thermostat=True, T_given=ts * s.meta["T"] * S.KB, freq_stat=4)
                step += 4
            alone.append(g.get_state()["x"])
    members = [_prepared(s, "fp64") for s in systems]
    try:
        with api.Batch(members) as b:
            step = 1
            for dt, ts in plan:
                opts = [api.md_opts(dt, thermostat=True, T_given=ts * s.meta["T"] * S.KB, freq_stat=4)
                        for s in systems]
                b.md_run(opts, 4, first_step=step)
                step += 4
        for k, g in enumerate(members):
            d = g.get_state()["x"] - alone[k]
            d -= systems[k].box * np.round(d / systems[k].box)
            assert np.abs(d).max() <= 1e-9, (k, np.abs(d).max())
    finally:
        for g in members:
            g.close()


def test_per_pass_and_per_system_batches_agree():
    """The per-pass graph (one launch per kernel of the step for all systems,
    batched FFT plans) against the per-system graph of the same members:
    positions within 1e-6 A after 8 mixed steps and far fewer launches."""
    systems = _members()
    runs = {}
    for mode in ("per_pass", "per_system"):
        members = [_prepared(s, "mixed") for s in systems]
        try:
            with api.Batch(members) as b:
                b.set_mode(mode)
                opts = [_opts(s) for s in systems]
                b.md_run(opts, 2, first_step=1)
                l0 = b.launch_count()
                b.md_run(opts, 6, first_step=3)
                assert b.mode() == mode
                runs[mode] = ([g.get_state()["x"] for g in members], (b.launch_count() - l0) / 6)
        finally:
            for g in members:
                g.close()
    for k, s in enumerate(systems):
        d = runs["per_pass"][0][k] - runs["per_system"][0][k]
        d -= s.box * np.round(d / s.box)
        assert np.abs(d).max() <= 1e-6, (k, np.abs(d).max())
    assert runs["per_pass"][1] < 0.6 * runs["per_system"][1], (runs["per_pass"][1], runs["per_system"][1])
