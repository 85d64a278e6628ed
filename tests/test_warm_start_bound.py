"""What a warm start can save, on the FP64 oracle (CPU): config 1's 32^3 cross-ply, one
unit load, Anderson depth 5, every warm-started solve stopped at 1e-6 times the COLD start's
first criterion (as the product's warm starts stop, `e0_ref` / `lsb_set_reference_e0`).

* The exact solution projected on its lowest 12^3 modes (the retained modes of the learned
  network: the best such a network could predict) starts ABOVE the cold start's criterion
  (the equilibrium residual sits at the phase interfaces, where the truncated field rings)
  and needs more updates than the cold start.
* The exact solution with white noise of 1e-4 of the field's variation halves the updates:
  a start has to be accurate to about that level, at full resolution, to pay.
"""

import numpy as np

from oracle import ls_oracle as O

N = 32


def _setup():
    from jaxmaterials_b200.data import fibres

    lm, mu = fibres.lame_fields(fibres.config_structure("c1", seed=0))
    return lm.astype(np.float64), mu.astype(np.float64), O.Grid(N, N, N, float(N), float(N), float(N))


def _lowpass(f, m):
    fh = np.fft.rfftn(f, axes=(-3, -2, -1))
    k = np.abs(np.fft.fftfreq(N, 1.0 / N))
    kz = np.arange(N // 2 + 1)
    keep = (k[:, None, None] < m / 2) & (k[None, :, None] < m / 2) & (kz[None, None, :] < m / 2)
    return np.fft.irfftn(fh * keep, s=(N, N, N), axes=(-3, -2, -1))


def test_warm_start_accuracy_bound():
    lm, mu, g = _setup()
    eb = np.array([1.0, 0.0, 0.0, 0.0, 0.0, 0.0])
    h = []
    _, _, cold = O.lippmann_schwinger(lm, mu, eb, g, rtol=1e-6, atol=1e-30, depth=5, maxiter=800,
                                      dtype=np.float64, history=h)
    e0 = h[0]
    exact, _, _ = O.lippmann_schwinger(lm, mu, eb, g, rtol=1e-13, atol=1e-40, depth=5,
                                       maxiter=3000, dtype=np.float64)

    def warm(start):
        hh = []
        _, _, it = O.lippmann_schwinger(lm, mu, eb, g, rtol=0.0, atol=1e-6 * e0, depth=5,
                                        maxiter=2000, dtype=np.float64, epsilon0=start, history=hh)
        return it, hh[0] / e0

    it12, c12 = warm(_lowpass(exact, 12))
    assert c12 > 1.0 and it12 >= cold, (it12, c12, cold)
    spread = np.abs(exact - eb[:, None, None, None]).max()
    noisy = exact + 1e-4 * spread * np.random.default_rng(1).standard_normal(exact.shape)
    itn, cn = warm(noisy)
    assert cn < 1e-2 and itn <= 0.6 * cold, (itn, cn, cold)
