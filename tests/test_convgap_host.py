"""Host side of the Conv + GAP fusion (no GPU): the weight scattering and the
conv index lists agree with the reference's goldens and the oracle, and the
plain model equals the sum-over-indices form the fusion relies on."""
import json
from pathlib import Path

import numpy as np

from oracle import convgap as OC

GD = Path(__file__).resolve().parent / "golden"


def test_scatter_matches_reference_goldens():
    from ckks_b200 import convgap as G
    d = np.load(GD / "golden_convgap.npz")
    m = json.load(open(GD / "golden_convgap.json"))
    for k in m["scatter"]:
        got = G.scatter_w(d[k + "_idx"], d[k + "_w"], m["scale"], m["q"], m["N"])
        assert np.array_equal(got, d[k + "_out"]), k


def test_conv_indices_and_plain_model():
    from ckks_b200 import convgap as G
    model = G.ConvGapModel.random(1)
    idx, vals = G.conv_gap_indices(model.conv_w[2, 0])
    assert (idx, vals) == OC.conv_gap_indices(model.conv_w[2, 0])
    # padding drops the taps of row / column -1 only: 13 border positions x 3 taps, 1 corner tap counted twice
    assert len(idx) == 49 * 9 - (2 * 7 * 3 - 1)
    x = np.random.default_rng(2).uniform(0, 1, (4, 784))
    direct = np.array([[sum(img[i] * v for i, v in zip(*G.conv_gap_indices(model.conv_w[f, 0]))) / 49
                        + model.conv_b[f] for f in range(4)] for img in x]) @ model.fc_w.T + model.fc_b
    assert np.max(np.abs(direct - model.plain_forward(x))) < 1e-12
