/* Fibre placement: jaxmaterials_b200/libfibres.so (host C++). The GPU voxelisation of the
 * placed fibres is lsb_voxelise_fibres in lippmann_schwinger.h.
 *
 * libfibres.so is a drop-in for the library the reference builds from
 * src/jaxmaterials/data/libfibres.cc and loads in
 * src/jaxmaterials/data/distributions_fibres.py:136-163: the first three functions keep
 * its names, arguments and results (bit for bit, with the same C++ runtime).
 */
#ifndef JAXMATERIALS_B200_FIBRES_H
#define JAXMATERIALS_B200_FIBRES_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces dist_periodic (libfibres.cc:31-47): dist[j] = minimum over the 3 x 3 periodic
 * images of |p + offset - q_j| in the box L[0] x L[1]; q holds n points (x, y) interleaved. */
void dist_periodic(const unsigned int n, const double p[2], const double *q, const double L[2],
                   double *dist);

/* Replaces initialise_rng (libfibres.cc:60-74): writes the textual state of a std::mt19937
 * seeded with `seed` into rng_state (no terminating NUL; the caller provides room for
 * 10000 bytes) and its length into *rng_state_length. */
void initialise_rng(unsigned int seed, unsigned int *rng_state_length, char *rng_state);

/* Replaces move_fibres (libfibres.cc:94-179): moves the n_fibres centres in
 * fibre_locations (x, y interleaved, in [0, domain_size]) by the random shaking algorithm
 * until num_repeats sweeps are done and the last sweep left every pair of fibres at least
 * eps_fibres apart (a fibre that finds no such place in it_max_ovlap trials takes its trial
 * with the fewest overlaps and forces another sweep). r_fibres: radii. The random stream
 * continues from, and is written back to, rng_state / *rng_state_length. n_fibres >= 3 (the
 * reference reads three nearest-neighbour distances). */
void move_fibres(const unsigned int n_fibres, const double *domain_size, const double *r_fibres,
                 double *fibre_locations, const unsigned int num_repeats, const double eps_fibres,
                 const unsigned int it_max_ovlap, unsigned int *rng_state_length, char *rng_state);

/* No reference counterpart: move_fibres on `nsets` independent fibre sets, each started
 * from a std::mt19937 seeded with `seed` (what the reference does for every layer: a new
 * FibreDistribution2d seeds its generator with the same constant,
 * distributions_fibres.py:165-172), on `threads` host threads (<= 0: all cores). Set i has
 * n_fibres[i] >= 3 fibres, box domain_sizes[2i..2i+1]; r_fibres and fibre_locations (x, y
 * interleaved) hold the sets one after another. Results equal nsets separate move_fibres
 * calls. max_sweeps > 0 stops a set after that many sweeps if it still has overlaps (the
 * reference sweeps on without bound, forever when the fibres do not fit); 0 = no bound.
 * Returns the number of sets stopped that way (0 = all placed), or -1 for invalid
 * arguments. */
int fibres_move_batch(int nsets, const unsigned int *n_fibres, const double *domain_sizes,
                      const double *r_fibres, double *fibre_locations, unsigned int num_repeats,
                      double eps_fibres, unsigned int it_max_ovlap, unsigned int seed,
                      unsigned int max_sweeps, int threads);

#ifdef __cplusplus
}
#endif

#endif /* JAXMATERIALS_B200_FIBRES_H */
