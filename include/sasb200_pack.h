/*
 * sasb200_pack.h -- C-ABI of libsasb200_pack.so: the values vectors of a fit
 * population expanded on the device from a compact per-set table.
 *
 * Reference interfaces replaced:
 *   sasb200_pack_values  make_kernel_args (sasmodels/details.py:225-254) with
 *                        the dispersity meshes of every distribution of the
 *                        plugin API (Dispersion._linspace and the gaussian,
 *                        uniform, rectangle, lognormal, schulz and boltzmann
 *                        _weights, get_weights: sasmodels/weights.py:21-220,
 *                        264-291) and the magnetic conversion
 *                        (convert_magnetism, details.py:288-306), for every
 *                        set of a population at once.  Set s's values
 *                        (val_size[s] doubles, a multiple of 32) are written
 *                        at values + val_off[s]:
 *                            scalars[s][0 .. nvalues), the nmag (M0, mtheta,
 *                              mphi) triples at its end turned into
 *                              (mx, my, mz) when magnetic[s] != 0
 *                            x of each kernel parameter k (npts[s][k] points,
 *                              or 1 when npts[s][k] == 0: idle)
 *                            the normalised weights in the same order
 *                            zeros up to val_size[s]
 *                        The value of kernel parameter k is scalars[s][2 + k];
 *                        widths/nsigmas[s][k] its dispersity width and number
 *                        of sigmas; kinds[s][k] its distribution (0 gaussian,
 *                        1 uniform, 2 rectangle, 3 lognormal, 4 schulz,
 *                        5 boltzmann); the points are those of index
 *                        first[s][k] .. first[s][k] + npts[s][k] - 1 of the
 *                        distribution's ntot[s][k]-point linspace (the ones
 *                        inside the parameter's limits); flags[k] bit 0:
 *                        width relative to the value (volume parameter),
 *                        bit 1: an idle parameter keeps its value (else 0,
 *                        an orientation jitter).  Sets with val_off[s] < 0
 *                        are skipped (marshaled on the host).
 *                        npars <= sasb200_pack_max_pars().
 * All arrays are device pointers; the call is asynchronous on *stream*.
 * Return 0, -1 for a bad argument, -3 for a launch error;
 * sasb200_pack_last_error() describes the last failure.
 */
#ifndef SASB200_PACK_H
#define SASB200_PACK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char *sasb200_pack_last_error(void);

int32_t sasb200_pack_max_pars(void);

int32_t sasb200_pack_values(int32_t n_sets, int32_t nvalues, int32_t npars, int32_t nmag,
                            const double *scalars, const double *widths,
                            const double *nsigmas, const int32_t *npts,
                            const int32_t *first, const int32_t *ntot,
                            const int32_t *kinds, const int32_t *flags,
                            const int32_t *magnetic, const int64_t *val_off,
                            const int64_t *val_size, double *values, void *stream);

#ifdef __cplusplus
}
#endif

#endif
