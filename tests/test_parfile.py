"""GSvit parameter files through gsvit_copy_b200.parfile: GSvit's own
self-test decks (written as make_test writes them, tests.c:93-268) parse into
the scene of plan.selftest_scene and step identically on the FP64 oracle;
GSvit's text output formats; keywords outside the path are refused."""
import os

import numpy as np
import pytest

from gsvit_copy_b200 import parfile, plan
from oracle.pyoracle import CpuSolver
from tests._selftest_deck import write_deck


@pytest.mark.parametrize("code", ["31111", "35011"])
def test_selftest_deck_is_the_selftest_scene(tmp_path, code):
    res = 64
    run = parfile.load_par(write_deck(str(tmp_path), res, code, 2 * res + 1))
    ref = plan.selftest_scene(code, res, 2 * res + 1)
    s = run.scene
    assert (s.xres, s.dx, s.dt, s.nsteps, s.matmode) == (ref.xres, ref.dx, ref.dt, ref.nsteps, ref.matmode)
    assert [bytes(m) for m in s.mats] == [bytes(m) for m in ref.mats]
    for name in ("mat", "epsilon", "sigma", "mu", "sigast"):
        a, b = getattr(s, name), getattr(ref, name)
        assert (a is None) == (b is None) and (a is None or np.array_equal(a, b)), name
    assert s.cpml == ref.cpml
    assert s.tsf["box"] == ref.tsf["box"] and np.array_equal(s.tsf["wave"], ref.tsf["wave"])
    assert (s.tsf["theta"], s.tsf["phi"], s.tsf["psi"]) == (ref.tsf["theta"], ref.tsf["phi"], ref.tsf["psi"])
    assert s.nfff["box"] == ref.nfff["box"]
    assert np.array_equal(s.nfff["points"], ref.nfff["points"]) and np.array_equal(s.nfff["istart"], ref.nfff["istart"])
    assert run.far_files == [f"{res}{code}"]


def test_parsed_deck_steps_like_the_scene_on_the_oracle(tmp_path):
    res, n = 64, 60
    run = parfile.load_par(write_deck(str(tmp_path), res, "35011", n))
    ref = plan.selftest_scene("35011", res, n)
    a, b = CpuSolver(run.scene), CpuSolver(ref)
    a.step(n)
    b.step(n)
    assert np.array_equal(a.nfff_series(), b.nfff_series())
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)


def test_text_outputs(tmp_path):
    deck = tmp_path / "d.par"
    deck.write_text("POOL\n30 30 30 1e-8 1e-8 1e-8\n\nCOMP\n20\n\nOUT_POINT\nAll 1 15 15 15 pall\n\n"
                    "OUT_POINT\nEy 1 10 11 12 pey\n\nOUT_IMAGE\nEx 20 15 -1 -1 img logscale\n\nVERBOSE\n3\n\n"
                    "BOUNDARY_ALL\ncpml 5 3 -1 0.03 4\n")
    run = parfile.load_par(str(deck))
    assert np.array_equal(run.scene.probes, [[15, 15, 15], [10, 11, 12]])
    probes = np.arange(2 * 20 * 6, dtype=np.float64).reshape(2, 20, 6) * 1.5e-3
    series = np.zeros((0, 3, 4))
    files = parfile.write_outputs(run, probes, series, 20, str(tmp_path))
    rows = open(tmp_path / "pall").read().splitlines()
    assert len(rows) == 19 and rows[2] == "2 %g %g %g %g %g %g" % tuple(probes[0, 2])
    assert open(tmp_path / "pey").read().splitlines()[5] == "5 %g" % probes[1, 5, 1]
    assert len(files) == 2


def test_far_field_log_is_minus_the_series(tmp_path):
    run = parfile.ParRun(scene=None, far_files=["ff"])
    series = np.random.default_rng(1).standard_normal((1, 3, 7))
    parfile.write_outputs(run, None, series, 7, str(tmp_path))
    back = np.loadtxt(tmp_path / "ff")
    assert np.array_equal(back[:, 0], np.arange(7))
    assert np.allclose(-back[:, 1:].T, series[0], rtol=1e-5)


@pytest.mark.parametrize("text,word", [("SOURCE_POINT\n1 1 1 0 f\n", "SOURCE_POINT"),
                                       ("BOUNDARY_ALL\nliao\n", "liao"),
                                       ("MEDIUM_LINEAR\nfile\n", "MEDIUM_LINEAR")])
def test_keywords_outside_the_path(tmp_path, text, word):
    deck = tmp_path / "x.par"
    deck.write_text("POOL\n20 20 20 1e-8 1e-8 1e-8\n\nCOMP\n10\n\n" + text)
    with pytest.raises(parfile.ParError, match=word):
        parfile.load_par(str(deck))


def test_killer_file_rule(tmp_path):
    """GSvit's killcheck (svit.c:91-107): stop when the file exists and reads 1."""
    from gsvit_copy_b200.run import killer_says_stop
    f = tmp_path / "killer"
    assert not killer_says_stop(str(f))            # absent
    for text, stop in (("0", False), ("2", False), ("1", True), ("  1\n", True), ("1 0", True), ("x1", False),
                       ("", False), ("-1", False)):
        f.write_text(text)
        assert killer_says_stop(str(f)) == stop, text


def test_killer_file_stops_the_step_loop(tmp_path):
    """The runner looks at the file after every `check_every` steps and stops
    cleanly once it says 1; without a killer file one call does all steps."""
    from gsvit_copy_b200.run import run_steps
    f = tmp_path / "killer"
    f.write_text("0")
    calls = []

    def step(k):
        calls.append(k)
        if sum(calls) >= 7:                      # an operator writes 1 after step 7
            f.write_text("1")

    assert run_steps(step, 100, str(f)) == 7 and calls == [1] * 7
    calls.clear()
    f.write_text("0")
    assert run_steps(step, 100, str(f), check_every=5) == 10 and calls == [5, 5]
    calls.clear()
    assert run_steps(step, 12, None) == 12 and calls == [12]
    calls.clear()
    f.write_text("0")
    assert run_steps(lambda k: calls.append(k), 9, str(f), check_every=4) == 9 and calls == [4, 4, 1]
