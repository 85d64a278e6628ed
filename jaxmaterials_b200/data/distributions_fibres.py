"""Fibre radius and 2-d fibre position distributions: the reference's
``src/jaxmaterials/data/distributions_fibres.py`` interface (``FibreRadiusDistribution``,
``FibreDistribution2d``) over the native ``libfibres.so`` (``include/fibres.h``).

Both classes take the reference's arguments and give its numbers: the radius draws use the
same NumPy generator calls (inverse transform of a normal density clipped to [r_min, r_max],
:26-72), the initial fibre lattice is built the same way (:102-118), and the shaking moves
(:174-203) run in ``libfibres.so``, which reproduces the reference's C++ library bit for bit.
The reference compiles its C++ with g++ every time a ``FibreDistribution2d`` is created; here
the library is built once with the package, and there is no fallback when it is missing
(the reference's NumPy shaking path, ``fast_code=False``, is not provided).

``place_batch`` moves many independent fibre sets in one call on all host cores.
"""

import ctypes
import itertools

import numpy as np
from scipy.stats import norm

from .. import _lib

__all__ = ["FibreRadiusDistribution", "FibreDistribution2d", "place_batch",
           "NUM_REPEATS", "IT_MAX_OVLAP", "EPS_FIBRES", "RNG_SEED"]

#: Shaking parameters used by the reference's iterator (distributions_fibres.py:176-178).
NUM_REPEATS = 30
IT_MAX_OVLAP = 5000
EPS_FIBRES = 3.0e-4
#: Seed of the C++ generator of every FibreDistribution2d (distributions_fibres.py:165).
RNG_SEED = 735283
_STATE_BYTES = 10000


class FibreRadiusDistribution:
    """Fibre radii: constant ``r_avg``, or (gaussian=True) normal with mean ``r_avg`` and
    standard deviation ``sigma`` restricted to [r_min, r_max], drawn by inverting its
    cumulative distribution tabulated at 1000 points (distributions_fibres.py:26-72)."""

    def __init__(self, r_avg, r_min, r_max, sigma, gaussian, seed=856219):
        self.r_avg = r_avg
        self.r_min = r_min
        self.r_max = r_max
        self.sigma = sigma
        self.gaussian = gaussian
        self._rng = np.random.default_rng(seed=seed)
        nodes = np.linspace(self.r_min, self.r_max, num=1000)
        cdf = np.cumsum(norm.pdf(nodes, loc=self.r_avg, scale=self.sigma))
        cdf /= cdf[-1]
        self._cdf = cdf
        self._x_cdf = np.linspace(0, 1, 1000)

    def draw(self, n_samples):
        """n_samples radii."""
        if not self.gaussian:
            return np.ones(shape=(n_samples,)) * self.r_avg
        xi = self._rng.uniform(low=0, high=1, size=n_samples)
        return np.interp(xi, self._cdf, self._x_cdf) * (self.r_max - self.r_min) + self.r_min


def initial_lattice(domain_size, r_avg, volume_fraction):
    """Regular start lattice of the shaking algorithm (distributions_fibres.py:102-118):
    ceil(L_d / r_avg * sqrt(vf / pi)) fibres along each direction, x-major order."""
    domain_size = np.asarray(domain_size, dtype=np.float64)
    per_dir = np.ceil(domain_size / r_avg * np.sqrt(volume_fraction / np.pi)).astype(np.int64)
    d = 2 * r_avg
    axes = (domain_size[k] * np.arange(0, (per_dir[k] - 0.5) * d, d) / (d * per_dir[k])
            for k in (0, 1))
    return np.asarray(list(itertools.product(*axes))).reshape([per_dir[0] * per_dir[1], 2])


def place_batch(domain_sizes, radii, locations, num_repeats=NUM_REPEATS, eps=EPS_FIBRES,
                it_max_ovlap=IT_MAX_OVLAP, seed=RNG_SEED, max_sweeps=0, threads=0):
    """Shake many independent fibre sets at once (``fibres_move_batch``).

    domain_sizes: (S, 2); radii: list of S arrays (n_i,); locations: list of S arrays
    (n_i, 2), start positions. Every set starts from a generator seeded with ``seed``, as
    each reference ``FibreDistribution2d`` does. Returns the list of moved positions.
    Raises if a set still overlaps after ``max_sweeps`` sweeps (> 0)."""
    lib = _lib.load_fibres()
    s = len(radii)
    counts = np.array([len(r) for r in radii], dtype=np.uint32)
    if s == 0:
        return []
    if np.any(counts < 3):
        raise ValueError("every fibre set needs at least 3 fibres")
    dom = np.ascontiguousarray(np.asarray(domain_sizes, dtype=np.float64).reshape(s, 2))
    rad = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64) for r in radii]))
    loc = np.ascontiguousarray(np.concatenate(
        [np.asarray(x, np.float64).reshape(-1, 2) for x in locations]))
    if loc.shape[0] != rad.shape[0]:
        raise ValueError("locations and radii differ in length")
    rc = lib.fibres_move_batch(
        s, counts.ctypes.data_as(_lib.c_uint_p), dom.ctypes.data_as(_lib.c_double_p),
        rad.ctypes.data_as(_lib.c_double_p), loc.ctypes.data_as(_lib.c_double_p),
        int(num_repeats), float(eps), int(it_max_ovlap), int(seed), int(max_sweeps),
        int(threads))
    if rc < 0:
        raise ValueError("fibres_move_batch: invalid arguments")
    if rc > 0:
        raise RuntimeError(f"{rc} fibre set(s) still overlap after {max_sweeps} sweeps")
    return np.split(loc, np.cumsum(counts)[:-1])


class FibreDistribution2d:
    """Fibres in a periodic 2-d box (distributions_fibres.py:75-295): iterating yields
    (positions (n, 2), radii (n,)), the regular start lattice shaken with freshly drawn radii.
    The C++ generator state persists across iterations of one instance, as in the
    reference. ``fast_code`` is accepted for the reference's signature; only the native
    path (True) exists."""

    def __init__(self, domain_size, volume_fraction=0.55,
                 r_fibre_dist=FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3,
                                                      r_max=10.0e-3, sigma=0.5e-3,
                                                      gaussian=True),
                 seed=141517, fast_code=True):
        self.domain_size = np.asarray(domain_size, dtype=np.float64)
        self._volume_fraction = volume_fraction
        self._r_fibre_dist = r_fibre_dist
        self._initial_fibre_locations = initial_lattice(self.domain_size, r_fibre_dist.r_avg,
                                                        volume_fraction)
        if not fast_code:
            raise ValueError("only the native shaking path (fast_code=True) is provided")
        self._lib = _lib.load_fibres()
        self._state_len = ctypes.c_uint()
        self._state = ctypes.create_string_buffer(_STATE_BYTES)
        self._lib.initialise_rng(RNG_SEED, ctypes.byref(self._state_len), self._state)

    def __iter__(self):
        while True:
            r = self._r_fibre_dist.draw(self._initial_fibre_locations.shape[0])
            x = np.array(self._initial_fibre_locations)
            r = np.ascontiguousarray(r, dtype=np.float64)
            x = np.ascontiguousarray(x, dtype=np.float64)
            self._lib.move_fibres(
                r.shape[0], self.domain_size.ctypes.data_as(_lib.c_double_p),
                r.ctypes.data_as(_lib.c_double_p), x.ctypes.data_as(_lib.c_double_p),
                NUM_REPEATS, EPS_FIBRES, IT_MAX_OVLAP, ctypes.byref(self._state_len),
                self._state)
            yield (x, r)
