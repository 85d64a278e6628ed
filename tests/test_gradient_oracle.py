"""The gradient identity used by the CUDA backward pass, pinned on the FP64 oracle:
for L(M), dL/dlambda(x) = sum_kl G_kl/w_l tr eps^k tr eps^l / N and
dL/dmu(x) = sum_kl G_kl/w_l 2 eps^k:eps^l / N with G = dL/dM, against central finite
differences (h = 1e-3 relative) of the oracle's effective stiffness."""

import numpy as np

from jaxmaterials_b200.data import fibres
from oracle import ls_oracle as O

W = np.array([1, 1, 1, 2, 2, 2.0])


def solve_all(lm, mu, g):
    eps, m = [], np.zeros((6, 6))
    for k in range(6):
        e = np.zeros(6)
        e[k] = 1.0
        ek, sk, _ = O.lippmann_schwinger(lm, mu, e, g, rtol=1e-13, atol=0.0, maxiter=3000,
                                         dtype=np.float64, depth=4, workers=1)
        eps.append(ek)
        m[k] = sk.mean(axis=(1, 2, 3))
    return m, np.array(eps)


def test_gradient_identity_vs_central_fd():
    st = fibres.generate_layered_fibres(12, 2, 2.0, 0.4, seed=3)
    lm, mu = fibres.lame_fields(st, dtype=np.float64)
    g = O.Grid(12, 12, 12, 12.0, 12.0, 12.0)
    m, e = solve_all(lm, mu, g)
    ct = m * (1 + 0.1 * np.random.default_rng(1).uniform(-1, 1, (6, 6)))
    loss = lambda mm: np.sum((mm - ct) ** 2)
    gw = 2 * (m - ct) / W[None, :]
    tr = e[:, 0] + e[:, 1] + e[:, 2]
    dot = np.einsum("kaxyz,laxyz,a->klxyz", e, e, W)
    n = g.number_of_voxels
    dl = np.einsum("kl,kxyz,lxyz->xyz", gw, tr, tr) / n
    dm = 2 * np.einsum("kl,klxyz->xyz", gw, dot) / n
    for v in [(0, 0, 0), (5, 7, 3), (11, 2, 9)]:
        for which, grad in (("lambda", dl), ("mu", dm)):
            arr = lm if which == "lambda" else mu
            h = 1e-3 * arr[v]
            p, q = arr.copy(), arr.copy()
            p[v] += h
            q[v] -= h
            if which == "lambda":
                fd = (loss(solve_all(p, mu, g)[0]) - loss(solve_all(q, mu, g)[0])) / (2 * h)
            else:
                fd = (loss(solve_all(lm, p, g)[0]) - loss(solve_all(lm, q, g)[0])) / (2 * h)
            assert abs(fd - grad[v]) <= 1e-5 * abs(fd) + 1e-12, (which, v, fd, grad[v])
