"""A GSvit self-test deck run unchanged through the front-end on the GPU
(python -m gsvit_copy_b200.run): the far-field log it writes against the
fixture pinned to GSvit's golden file (relative L2 1e-5; the log holds %g
text, 6 significant digits)."""
import os

import numpy as np
import pytest

from gsvit_copy_b200 import run as runner
from tests._selftest_deck import write_deck
from tests._util import rel_l2

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_selftest_deck_far_field_log(tmp_path):
    g0 = np.load(os.path.join(GOLD, "selftest_20035011.npz"))
    n = int(g0["nsteps"])
    deck = write_deck(str(tmp_path), 200, "35011", n)
    assert runner.main([deck, "--outdir", str(tmp_path)]) == 0
    log = np.loadtxt(os.path.join(str(tmp_path), "20035011"))
    series = -log[:, 1:].T
    ref = g0["series"]
    assert series.shape == ref.shape
    assert rel_l2(series, ref) < 1e-5, rel_l2(series, ref)
