// Fibre placement by random shaking (host C++), a drop-in for the reference's
// libfibres.so (src/jaxmaterials/data/libfibres.cc:31-179, loaded by
// src/jaxmaterials/data/distributions_fibres.py:136-163): the same three C entry points
// with the same arguments and results, plus a batched entry point that moves many
// independent fibre sets (layers of many samples) on all host cores.
//
// The algorithm is sequential Monte Carlo: every trial position of a fibre depends on the
// positions accepted before it, and the trials consume one random stream in order. Its
// results are reproduced bit for bit (the same std::mt19937 stream, the same
// std::shuffle / std::uniform_real_distribution and libm cos/sin as the reference's
// library built with the same C++ runtime), so it stays on the host; the parallel work
// of a dataset (independent layers and samples) is spread over threads, and the
// voxelisation of the placed fibres runs on the GPU (voxelise.cu).
#include "../../include/fibres.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace {

// Squared minimum-image distance over the 3 x 3 periodic copies, in the reference's
// evaluation order (offsets x then y in -1, 0, 1; libfibres.cc:34-45).
inline double min_image_d2(const double* p, const double* q, const double* L) {
  double d2_min = 4.0 * L[0] * L[1];
  for (int ox = -1; ox <= 1; ++ox)
    for (int oy = -1; oy <= 1; ++oy) {
      const double dx = p[0] + L[0] * ox - q[0];
      const double dy = p[1] + L[1] * oy - q[1];
      const double d2 = dx * dx + dy * dy;
      d2_min = d2 < d2_min ? d2 : d2_min;
    }
  return d2_min;
}

void distances(unsigned n, const double* p, const double* q, const double* L, double* dist) {
  for (unsigned j = 0; j < n; ++j) dist[j] = std::sqrt(min_image_d2(p, q + 2 * j, L));
}

// One call of the shaking algorithm on one fibre set (libfibres.cc:94-169):
// labels shuffled once; sweeps over the fibres in label order until num_repeats sweeps
// are done and the last sweep placed every fibre without overlap. A fibre's trial
// positions are drawn uniformly in a disc (radius = mean distance to its three nearest
// neighbours) around its current centre until the gap to every other fibre is at least
// eps; after it_max_ovlap failed trials the trial with the fewest overlaps is kept.
// Returns false when max_sweeps (> 0) sweeps ended with overlaps left (the reference has no
// such bound: it sweeps until a sweep succeeds, which never happens for a packing that
// leaves no room).
bool shake(std::mt19937& rng, unsigned n, const double* L, const double* r, double* loc,
           unsigned num_repeats, double eps, unsigned it_max_ovlap, unsigned max_sweeps = 0) {
  std::vector<unsigned> labels(n);
  std::iota(labels.begin(), labels.end(), 0u);
  std::shuffle(labels.begin(), labels.end(), rng);
  std::vector<double> dist(n);
  std::uniform_real_distribution<double> uniform(0.0, 1.0);
  const double self_gap = L[0] + L[1];
  bool overlap = true;
  for (unsigned sweep = 0; overlap || sweep < num_repeats; ++sweep) {
    if (max_sweeps > 0 && sweep >= max_sweeps) return false;
    overlap = false;
    for (unsigned jj = 0; jj < n; ++jj) {
      const unsigned me = labels[jj];
      const double p[2] = {loc[2 * me], loc[2 * me + 1]};
      const double r_me = r[me];
      distances(n, p, loc, L, dist.data());
      dist[me] = self_gap;
      // mean of the three smallest distances, summed in ascending order
      const unsigned k3 = n < 3 ? n : 3;
      std::partial_sort(dist.begin(), dist.begin() + k3, dist.end());
      double s = 0.0;
      for (unsigned i = 0; i < k3; ++i) s += dist[i];
      const double radius = s / 3.0;
      double gap = 0.0;
      unsigned trials = 0, best_overlaps = n + 1;
      double best[2] = {p[0], p[1]};
      double trial[2] = {p[0], p[1]};
      while (gap < eps) {
        const double u_r = radius * uniform(rng);
        const double u_t = 2 * M_PI * uniform(rng);
        trial[0] = p[0] + u_r * std::cos(u_t);
        trial[1] = p[1] + u_r * std::sin(u_t);
        for (int d = 0; d < 2; ++d) {
          while (trial[d] < 0) trial[d] += L[d];
          while (trial[d] > L[d]) trial[d] -= L[d];
        }
        distances(n, trial, loc, L, dist.data());
        dist[me] = self_gap;
        unsigned overlaps = 0;
        for (unsigned i = 0; i < n; ++i) {
          dist[i] -= r_me + r[i];
          overlaps += dist[i] < 0;
        }
        gap = *std::min_element(dist.begin(), dist.end());
        if (overlaps < best_overlaps) {
          best[0] = trial[0];
          best[1] = trial[1];
          best_overlaps = overlaps;
        }
        if (++trials > it_max_ovlap) {
          trial[0] = best[0];
          trial[1] = best[1];
          overlap = true;
          break;
        }
      }
      loc[2 * me] = trial[0];
      loc[2 * me + 1] = trial[1];
    }
  }
  return true;
}

void write_state(const std::mt19937& rng, unsigned int* len, char* state) {
  std::ostringstream os;
  os << rng;
  const std::string s = os.str();
  *len = (unsigned)s.size();
  std::memcpy(state, s.data(), s.size());
}

bool read_state(std::mt19937& rng, unsigned len, const char* state) {
  std::istringstream is(std::string(state, len));
  is >> rng;
  return !is.fail();
}

}  // namespace

extern "C" {

void dist_periodic(const unsigned int n, const double p[2], const double* q, const double L[2],
                   double* dist) {
  distances(n, p, q, L, dist);
}

void initialise_rng(unsigned int seed, unsigned int* rng_state_length, char* rng_state) {
  std::mt19937 rng;
  rng.seed(seed);
  write_state(rng, rng_state_length, rng_state);
}

void move_fibres(const unsigned int n_fibres, const double* domain_size, const double* r_fibres,
                 double* fibre_locations, const unsigned int num_repeats, const double eps_fibres,
                 const unsigned int it_max_ovlap, unsigned int* rng_state_length, char* rng_state) {
  std::mt19937 rng;
  read_state(rng, *rng_state_length, rng_state);
  shake(rng, n_fibres, domain_size, r_fibres, fibre_locations, num_repeats, eps_fibres,
        it_max_ovlap);
  write_state(rng, rng_state_length, rng_state);
}

int fibres_move_batch(int nsets, const unsigned int* n_fibres, const double* domain_sizes,
                      const double* r_fibres, double* fibre_locations, unsigned int num_repeats,
                      double eps_fibres, unsigned int it_max_ovlap, unsigned int seed,
                      unsigned int max_sweeps, int threads) {
  if (nsets < 0 || (nsets > 0 && (!n_fibres || !domain_sizes || !r_fibres || !fibre_locations)))
    return -1;
  std::vector<size_t> off(nsets + 1, 0);
  for (int i = 0; i < nsets; ++i) {
    if (n_fibres[i] < 3) return -1;
    off[i + 1] = off[i] + n_fibres[i];
  }
  for (int i = 0; i < nsets; ++i)
    if (!(domain_sizes[2 * i] > 0.0) || !(domain_sizes[2 * i + 1] > 0.0)) return -1;
  unsigned hw = std::thread::hardware_concurrency();
  int nt = threads > 0 ? threads : (int)(hw ? hw : 1);
  nt = std::max(1, std::min(nt, nsets));
  std::vector<int> unfinished(nt, 0);
  auto work = [&](int t) {
    for (int i = t; i < nsets; i += nt) {
      std::mt19937 rng;
      rng.seed(seed);
      if (!shake(rng, n_fibres[i], domain_sizes + 2 * i, r_fibres + off[i],
                 fibre_locations + 2 * off[i], num_repeats, eps_fibres, it_max_ovlap, max_sweeps))
        ++unfinished[t];
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  return std::accumulate(unfinished.begin(), unfinished.end(), 0);
}

}  // extern "C"
