"""Chi-squared consistency of sampled shots with exact probabilities."""
import numpy as np
from scipy import stats


def chi2_ok(samples, probs, shots, alpha=1e-4, min_expected=5.0):
    """Bins with at least `min_expected` expected counts are kept, the rest are
    merged into one bin; True if the chi-squared p-value exceeds alpha."""
    probs = np.asarray(probs, dtype=np.float64)
    probs = probs / probs.sum()
    counts = np.bincount(np.asarray(samples, dtype=np.int64), minlength=probs.size).astype(np.float64)
    exp = probs * shots
    big = exp >= min_expected
    obs_b, exp_b = counts[big], exp[big]
    rest_o, rest_e = counts[~big].sum(), exp[~big].sum()
    if rest_e > 0:
        obs_b = np.append(obs_b, rest_o)
        exp_b = np.append(exp_b, rest_e)
    if obs_b.size < 2:
        return True
    chi = float(((obs_b - exp_b) ** 2 / exp_b).sum())
    p = stats.chi2.sf(chi, obs_b.size - 1)
    return p > alpha
