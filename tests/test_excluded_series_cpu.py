"""The small-argument series the excluded-pair correction kernel uses for
h(x) = (erf(x) - 2/sqrt(pi) x exp(-x^2)) / x^3 (x = beta r below 0.7): its
eight terms, evaluated in FP64, against the closed form (well below FP32
rounding)."""
import numpy as np
from scipy.special import erf


def test_series_matches_closed_form():
    x = np.linspace(0.05, 0.7, 200)
    closed = (erf(x) - 2.0 / np.sqrt(np.pi) * x * np.exp(-x * x)) / x ** 3
    x2 = x * x
    coeffs = [2.0 / 3.0, -0.4, 1.0 / 7.0, -1.0 / 27.0, 1.0 / 132.0, -1.0 / 780.0, 1.0 / 5400.0, -1.0 / 42840.0]
    series = 2.0 / np.sqrt(np.pi) * sum(c * x2 ** k for k, c in enumerate(coeffs))
    assert np.abs(series / closed - 1.0).max() < 3e-8
