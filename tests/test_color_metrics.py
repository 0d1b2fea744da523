"""CIEDE2000 of the precision reports (oracle/color.py) on pairs from the supplementary
test data of Sharma, Wu and Dalal (Color Research & Application 30(1), 2005), and the
sRGB -> CIELAB conversion on its anchor points. No GPU."""
import numpy as np

from oracle import color

PAIRS = [
    ((50.0000, 2.6772, -79.7751), (50.0000, 0.0000, -82.7485), 2.0425),
    ((50.0000, 3.1571, -77.2803), (50.0000, 0.0000, -82.7485), 2.8615),
    ((50.0000, 2.8361, -74.0200), (50.0000, 0.0000, -82.7485), 3.4412),
    ((50.0000, 0.0000, 0.0000), (50.0000, -1.0000, 2.0000), 2.3669),
    ((50.0000, 2.5000, 0.0000), (73.0000, 25.0000, -18.0000), 27.1492),
    ((60.2574, -34.0099, 36.2677), (60.4626, -34.1751, 39.4387), 1.2644),
]


def test_ciede2000_reference_pairs():
    a = np.array([p[0] for p in PAIRS])
    b = np.array([p[1] for p in PAIRS])
    want = np.array([p[2] for p in PAIRS])
    np.testing.assert_allclose(color.delta_e2000(a, b), want, atol=1e-4)
    np.testing.assert_allclose(color.delta_e2000(b, a), want, atol=1e-4)


def test_srgb_anchor_points():
    lab = color.srgb_encoded_to_lab(np.array([[1.0, 1.0, 1.0], [0.0, 0.0, 0.0], [1.0, 0.0, 0.0]]))
    np.testing.assert_allclose(lab[0], [100.0, 0.0, 0.0], atol=1e-3)
    np.testing.assert_allclose(lab[1], [0.0, 0.0, 0.0], atol=1e-9)
    np.testing.assert_allclose(lab[2], [53.24, 80.09, 67.20], atol=0.02)
    s = color.delta_e_stats(np.full((4, 4, 3), 0.5), np.full((4, 4, 3), 0.5))
    assert s == {"p50": 0.0, "p99": 0.0, "max": 0.0}
