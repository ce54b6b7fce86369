"""Initialisation strategies of the reference front end
(pyaugur/pyaugur/augurdistlib.py:23-36) and the initial-point values they
give per distribution (augurdistlib.py:40-168): AugurDefault uses fixed
values (Dirichlet: uniform; Normal: its mean; Exponential: 1; InvGamma: 0.5;
Categorical: 0; MvNormal: zeros; InvWishart: identity), AugurRandom draws
from the prior, AugurUser takes the caller's point."""
import numpy as np


class AugurInitStrat(object):
    pass


class AugurRandom(AugurInitStrat):
    pass


class AugurDefault(AugurInitStrat):
    pass


class AugurUser(AugurInitStrat):
    def __init__(self, initPt):
        self.initPt = initPt


def init_value(strat, dist, args, rng):
    """Initial value of one parameter with distribution `dist` and evaluated
    arguments `args`."""
    random = isinstance(strat, AugurRandom)
    if dist == "Dirichlet":
        a = np.asarray(args[0], np.float64)
        return rng.dirichlet(a) if random else np.full(len(a), 1.0 / len(a))
    if dist == "Normal":
        mean, var = args
        return float(rng.normal(mean, np.sqrt(var))) if random else float(mean)
    if dist == "Exponential":
        return float(rng.exponential(1.0 / args[0])) if random else 1.0
    if dist == "InvGamma":
        shape, scale = args
        return float(1.0 / rng.gamma(shape, 1.0 / scale)) if random else 0.5
    if dist == "Categorical":
        pmf = np.asarray(args[0], np.float64)
        return int(np.searchsorted(np.cumsum(pmf), rng.uniform(0, pmf.sum()))) if random else 0
    if dist == "MvNormal":
        mu, cov = np.asarray(args[0], np.float64), np.asarray(args[1], np.float64)
        return rng.multivariate_normal(mu, cov) if random else np.zeros(len(mu))
    if dist == "InvWishart":
        df, scale = int(args[0]), np.asarray(args[1], np.float64)
        if not random:
            return np.eye(scale.shape[0])
        A = rng.multivariate_normal(np.zeros(scale.shape[0]), np.linalg.inv(scale), size=df)
        return np.linalg.inv(A.T @ A)
    raise NotImplementedError("no initialiser for %s" % dist)
