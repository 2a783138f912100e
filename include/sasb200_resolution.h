/*
 * sasb200_resolution.h -- C-ABI of libsasb200_resolution.so: resolution
 * smearing of a theory curve that is already on the device.
 *
 * Reference interfaces replaced:
 *   sasb200_pinhole_smear      Pinhole1D.apply -> apply_resolution_matrix
 *                              with the matrix of pinhole_resolution
 *                              (sasmodels/resolution.py:109-110, 172-220);
 *                              here the band of calculated points of each
 *                              measured q (lo[i] <= j < hi[i]) replaces the
 *                              dense n_calc x nq matrix and the weights are
 *                              formed on the fly from the bin edges.
 *   sasb200_slit_smear         Slit1D.apply with the matrix of
 *                              slit_resolution (sasmodels/resolution.py:
 *                              168-169, 223-395); q_calc is the signed,
 *                              sorted calculation grid, n_length the steps
 *                              across the slit width (30 in the reference).
 *   sasb200_pinhole_smear_sets the pinhole smearing of n_sets curves (a fit
 *                              population on one data set) in one launch.
 *   sasb200_nllf_sets          Experiment.nllf of every curve against one
 *                              data set: 0.5 sum(((theory - Iq)/dIq)^2)
 *                              (sasmodels/bumps_model.py:263-282).
 *   sasb200_pinhole2d_average  Pinhole2D.apply (sasmodels/resolution2d.py:
 *                              162-175): np.average over the oversampling
 *                              bins, theory laid out bin-major [nbins][nq],
 *                              wsum = the sum of the bin weights.
 * All arrays are device pointers; the calls are asynchronous on *stream*.
 * Return 0, -1 for a bad argument, -3 for a launch error;
 * sasb200_resolution_last_error() describes the last failure.
 */
#ifndef SASB200_RESOLUTION_H
#define SASB200_RESOLUTION_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char *sasb200_resolution_last_error(void);

int32_t sasb200_pinhole_smear(int32_t nq, int32_t n_calc, const double *q, const double *width,
                              const int32_t *lo, const int32_t *hi, const double *edges,
                              const double *theory, double *out, void *stream);

int32_t sasb200_pinhole_smear_sets(int32_t n_sets, int32_t nq, int32_t n_calc, const double *q,
                                   const double *width, const int32_t *lo, const int32_t *hi,
                                   const double *edges, const double *theory,
                                   int64_t theory_stride, double *out, int64_t out_stride,
                                   void *stream);

int32_t sasb200_nllf_sets(int32_t n_sets, int32_t nq, const double *theory,
                          int64_t theory_stride, const double *y, const double *dy,
                          double *out, void *stream);

int32_t sasb200_slit_smear(int32_t nq, int32_t n_calc, const double *q, const double *width,
                           const double *length, int32_t n_length, const double *q_calc,
                           const double *edges, const double *theory, double *out,
                           void *stream);

int32_t sasb200_pinhole2d_average(int32_t nq, int32_t nbins, const double *theory,
                                  const double *weights, double wsum, double *out,
                                  void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SASB200_RESOLUTION_H */
