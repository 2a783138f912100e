"""
Resolution smearing with the smearing itself on the GPU.

Mirrors the reference's resolution classes (``sasmodels/resolution.py``
Perfect1D, Pinhole1D, Slit1D; ``sasmodels/resolution2d.py`` Pinhole2D): the
same constructor arguments, the same
``q``/``q_calc`` attributes and the same ``apply(theory)``, so a caller that
builds ``Pinhole1D(q, dq)`` (or ``Pinhole2D(data)``), evaluates the model at
``q_calc`` and calls ``apply`` gets the same smeared curve.  ``apply`` takes
either a host array or a CUDA tensor (e.g. ``B200Kernel.Iq_device``) and
returns the same kind, so theory and smearing stay on the device.

The 1D smearing never forms the dense n_calc x nq weight matrix: each
measured q only sees the calculated points inside its +2.5/-3 sigma window
(``resolution.py:206-216``), found here once by binary search, and the GPU
forms the gaussian bin weights of that band on the fly
(``csrc/resolution.cu``).  ``weight_matrix`` is still available for callers
that read it, built on the host on first access.
"""

import ctypes as ct
import os

import numpy as np

from ._abi import LIB_DIR

MINIMUM_RESOLUTION = 1e-8
MINIMUM_ABSOLUTE_Q = 0.02
PINHOLE_N_SIGMA = (2.5, 3.0)
#: 2D: singular widths are raised to this; oversampling of the polar
#: resolution cell per accuracy level (resolution2d.py:14-21)
SIGMA_ZERO = 1.0e-010
NSIGMA_2D = 3.0
NR = {'xhigh': 10, 'high': 5, 'med': 5, 'low': 3}
NPHI = {'xhigh': 20, 'high': 12, 'med': 6, 'low': 4}

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(LIB_DIR, "libsasb200_resolution.so")
        if not os.path.exists(path):
            raise RuntimeError("resolution library not built: %s" % path)
        lib = ct.CDLL(path)
        P, I = ct.c_void_p, ct.c_int32
        lib.sasb200_pinhole_smear.argtypes = [I, I, P, P, P, P, P, P, P, P]
        lib.sasb200_pinhole_smear.restype = I
        lib.sasb200_pinhole2d_average.argtypes = [I, I, P, P, ct.c_double, P, P]
        lib.sasb200_slit_smear.argtypes = [I, I, P, P, P, I, P, P, P, P, P]
        lib.sasb200_slit_smear.restype = I
        L = ct.c_int64
        lib.sasb200_pinhole_smear_sets.argtypes = [I, I, I, P, P, P, P, P, P, L, P, L, P]
        lib.sasb200_pinhole_smear_sets.restype = I
        lib.sasb200_nllf_sets.argtypes = [I, I, P, L, P, P, P, P]
        lib.sasb200_nllf_sets.restype = I
        lib.sasb200_pinhole2d_average.restype = I
        lib.sasb200_resolution_last_error.restype = ct.c_char_p
        _LIB = lib
    return _LIB


def _check(status, what):
    if status != 0:
        raise RuntimeError("%s failed (%d): %s"
                           % (what, status, _lib().sasb200_resolution_last_error().decode()))


# ---------------------------------------------------------------- q grids --
def bin_edges(x):
    """Edges half way between bin centres, the end bins mirrored
    (``resolution.py:423-438``)."""
    x = np.asarray(x, 'd')
    if len(x) < 2 or (np.diff(x) < 0).any():
        raise ValueError("Expected bins to be an increasing set")
    return np.hstack([x[0] - 0.5*(x[1] - x[0]), 0.5*(x[1:] + x[:-1]),
                      x[-1] + 0.5*(x[-1] - x[-2])])


def linear_extrapolation(q, q_min, q_max):
    """Extend sorted q to [q_min, q_max] with steps like the end intervals
    (``resolution.py:460-482``); extrapolated values may be negative."""
    q = np.sort(q)
    if q_min + 2*MINIMUM_RESOLUTION < q[0]:
        delta = q[1] - q[0] if len(q) > 1 else 0
        n_low = int(np.ceil((q[0] - q_min)/delta)) if delta > 0 else 15
        q_low = np.linspace(q_min, q[0], n_low + 1)[:-1]
    else:
        q_low = []
    if q_max - 2*MINIMUM_RESOLUTION > q[-1]:
        delta = q[-1] - q[-2] if len(q) > 1 else 0
        n_high = int(np.ceil((q_max - q[-1])/delta)) if delta > 0 else 15
        q_high = np.linspace(q[-1], q_max, n_high + 1)[1:]
    else:
        q_high = []
    return np.concatenate([q_low, q, q_high])


def _nsigma(nsigma):
    try:
        lo, hi = nsigma
    except TypeError:
        lo = hi = nsigma
    return lo, hi


def pinhole_extend_q(q, q_width, nsigma=PINHOLE_N_SIGMA):
    """Calculation points covering every q's window (``resolution.py:398-409``)."""
    lo, hi = _nsigma(nsigma)
    q_min, q_max = np.min(q - lo*q_width), np.max(q + hi*q_width)
    return linear_extrapolation(q, q_min, q_max)


def geometric_extrapolation(q, q_min, q_max, points_per_decade=None):
    """Extend sorted q to [q_min, q_max] with geometric steps like the data's
    average step (``resolution.py:485-543``)."""
    q = np.sort(q)
    data_min, data_max = q[0], q[-1]
    if points_per_decade is None:
        if data_max > data_min:
            log_delta_q = (np.log(data_max) - np.log(data_min))/(len(q) - 1)
        else:
            log_delta_q = np.log(10.)/10
    else:
        log_delta_q = np.log(10.)/points_per_decade
    if q_min < data_min:
        if q_min < 0:
            q_min = data_min*MINIMUM_ABSOLUTE_Q
        n_low = int(np.ceil((np.log(q[0]) - np.log(q_min))/log_delta_q))
        q_low = np.logspace(np.log10(q_min), np.log10(q[0]), n_low + 1)[:-1]
    else:
        q_low = []
    if q_max > data_max:
        n_high = int(np.ceil((np.log(q_max) - np.log(data_max))/log_delta_q))
        q_high = np.logspace(np.log10(data_max), np.log10(q_max), n_high + 1)[1:]
    else:
        q_high = []
    return np.concatenate([q_low, q, q_high])


def slit_extend_q(q, q_length=0, q_width=0):
    """Calculation points for slit smearing (``resolution.py:412-420``)."""
    q_min = np.min(q - q_width)
    q_max = np.max(np.sqrt((q + q_width)**2 + q_length**2))
    return geometric_extrapolation(q, q_min, q_max)


def _device(device):
    import torch
    dev = torch.device(device if device is not None else "cuda")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


class Perfect1D:
    """No smearing (``resolution.py:52-63``)."""

    def __init__(self, q):
        self.q_calc = self.q = q

    def apply(self, theory):
        return theory


class Pinhole1D:
    """
    Pinhole aperture with q-dependent gaussian resolution
    (``resolution.py:66-110``): *q* measured points, *q_width* their 1-sigma
    widths, *q_calc* the calculation points (estimated when None).
    """

    def __init__(self, q, q_width, q_calc=None, nsigma=PINHOLE_N_SIGMA, device=None):
        self.q, self.q_width = q, q_width
        q = np.asarray(q, 'd')
        q_calc = (pinhole_extend_q(q, q_width, nsigma=nsigma)
                  if q_calc is None else np.sort(q_calc))
        # models may be undefined at very low |q|
        q_calc = q_calc[abs(q_calc) >= MINIMUM_ABSOLUTE_Q*np.min(q)]
        width = np.maximum(np.broadcast_to(np.asarray(q_width, 'd'), q.shape),
                           MINIMUM_RESOLUTION)
        lo_s, hi_s = _nsigma(nsigma)
        self._signed_q_calc = q_calc
        self._width = np.ascontiguousarray(width)
        self._nsigma = (lo_s, hi_s)
        self.edges = bin_edges(q_calc)
        # band of each q: calculated points inside [q - lo s, q + hi s]
        self.band_lo = np.searchsorted(q_calc, q - lo_s*width, side="left").astype(np.int32)
        self.band_hi = np.searchsorted(q_calc, q + hi_s*width, side="right").astype(np.int32)
        self.q_calc = abs(q_calc)
        self._device_arg = device
        self._dev = None
        self._weight_matrix = None

    @property
    def device(self):
        return _device(self._device_arg)

    def _upload(self):
        if self._dev is None:
            import torch
            d = dict(device=self.device)
            self._dev = dict(
                q=torch.as_tensor(np.ascontiguousarray(self.q, 'd'), **d),
                width=torch.as_tensor(self._width, **d),
                lo=torch.as_tensor(self.band_lo, **d), hi=torch.as_tensor(self.band_hi, **d),
                edges=torch.as_tensor(self.edges, **d))
        return self._dev

    def apply(self, theory, stream=None):
        """Smeared I(q) from I(q_calc): a CUDA tensor in, a CUDA tensor out
        (enqueued on *stream*, default the current stream); a host array in,
        a host array out."""
        import torch
        on_device = isinstance(theory, torch.Tensor) and theory.is_cuda
        t = (theory if on_device else
             torch.as_tensor(np.ascontiguousarray(theory, 'd'), device=self.device))
        t = t.to(torch.float64).contiguous()
        if t.numel() != len(self.q_calc):
            raise ValueError("theory has %d points, q_calc %d" % (t.numel(), len(self.q_calc)))
        d = self._upload()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(st):
            out = torch.empty(len(d["q"]), dtype=torch.float64, device=self.device)
            _check(_lib().sasb200_pinhole_smear(
                len(d["q"]), t.numel(), d["q"].data_ptr(), d["width"].data_ptr(),
                d["lo"].data_ptr(), d["hi"].data_ptr(), d["edges"].data_ptr(), t.data_ptr(),
                out.data_ptr(), st.cuda_stream), "pinhole_smear")
        if on_device:
            return out
        st.synchronize()
        return out.cpu().numpy()

    def apply_sets(self, theory, stream):
        """Smear many curves at once: *theory* a CUDA tensor [n_sets, n_calc]
        (rows contiguous), result [n_sets, nq] on the device, on *stream*."""
        import torch
        n_sets, n_calc = theory.shape
        if n_calc != len(self.q_calc) or theory.stride(1) != 1:
            raise ValueError("theory must be [n_sets, %d] with contiguous rows" % len(self.q_calc))
        d = self._upload()
        nq = len(d["q"])
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            out = torch.empty((n_sets, nq), dtype=torch.float64, device=self.device)
            _check(_lib().sasb200_pinhole_smear_sets(
                n_sets, nq, n_calc, d["q"].data_ptr(), d["width"].data_ptr(),
                d["lo"].data_ptr(), d["hi"].data_ptr(), d["edges"].data_ptr(),
                theory.data_ptr(), theory.stride(0), out.data_ptr(), nq, stream.cuda_stream),
                "pinhole_smear_sets")
        return out

    @property
    def weight_matrix(self):
        """Dense n_calc x nq weights (``resolution.py:182-220``), on the host;
        only for callers that read the matrix itself."""
        if self._weight_matrix is None:
            from scipy.special import erf
            q = np.asarray(self.q, 'd')
            cdf = erf((self.edges[:, None] - q[None, :])/(np.sqrt(2.0)*self._width)[None, :])
            w = cdf[1:] - cdf[:-1]
            lo_s, hi_s = self._nsigma
            qc = self._signed_q_calc
            w[qc[:, None] < (q - lo_s*self._width)[None, :]] = 0.
            w[qc[:, None] > (q + hi_s*self._width)[None, :]] = 0.
            w /= np.sum(w, axis=0)[None, :]
            self._weight_matrix = w
        return self._weight_matrix


class Slit1D:
    """
    Slit aperture smearing (``resolution.py:113-169``): *q_length* along the
    slit, *q_width* across it (scalars or per point); *q_calc* estimated when
    None.  A nonzero width with a zero length is refused, as by the
    reference.
    """

    N_LENGTH = 30

    def __init__(self, q, q_length=None, q_width=None, q_calc=None, device=None):
        self.q_length, self.q_width = q_length, q_width
        n = len(q)
        width = (np.zeros(n) if q_width is None else
                 np.ones(n)*q_width if np.isscalar(q_width) else np.asarray(q_width, 'd'))
        length = (np.zeros(n) if q_length is None else
                  np.ones(n)*q_length if np.isscalar(q_length) else np.asarray(q_length, 'd'))
        if np.any((width != 0) & (length == 0)):
            raise NotImplementedError("We do not yet handle the q_length=0.0 case for all "
                                      "q_width.")
        self.q = np.asarray(q, 'd').flatten()
        q_calc = (slit_extend_q(q, q_length=length, q_width=width)
                  if q_calc is None else np.sort(q_calc))
        q_calc = q_calc[abs(q_calc) >= MINIMUM_ABSOLUTE_Q*np.min(self.q)]
        self._signed_q_calc = q_calc
        self._width = np.ascontiguousarray(width, 'd')
        self._length = np.ascontiguousarray(length, 'd')
        self.edges = bin_edges(q_calc)
        self.q_calc = abs(q_calc)
        self._device_arg = device
        self._dev = None

    @property
    def device(self):
        return _device(self._device_arg)

    def apply(self, theory, stream=None):
        """Smeared I(q) from I(q_calc); CUDA tensor in -> CUDA tensor out,
        host array in -> host array out."""
        import torch
        on_device = isinstance(theory, torch.Tensor) and theory.is_cuda
        t = (theory if on_device else
             torch.as_tensor(np.ascontiguousarray(theory, 'd'), device=self.device))
        t = t.to(torch.float64).contiguous()
        if t.numel() != len(self.q_calc):
            raise ValueError("theory has %d points, q_calc %d" % (t.numel(), len(self.q_calc)))
        if self._dev is None:
            d = dict(device=self.device)
            self._dev = dict(q=torch.as_tensor(self.q, **d), w=torch.as_tensor(self._width, **d),
                             l=torch.as_tensor(self._length, **d),
                             qc=torch.as_tensor(np.ascontiguousarray(self._signed_q_calc), **d),
                             e=torch.as_tensor(self.edges, **d))
        d = self._dev
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(st):
            out = torch.empty(len(self.q), dtype=torch.float64, device=self.device)
            _check(_lib().sasb200_slit_smear(
                len(self.q), t.numel(), d["q"].data_ptr(), d["w"].data_ptr(),
                d["l"].data_ptr(), self.N_LENGTH, d["qc"].data_ptr(), d["e"].data_ptr(),
                t.data_ptr(), out.data_ptr(), st.cuda_stream), "slit_smear")
        if on_device:
            return out
        st.synchronize()
        return out.cpu().numpy()


class Pinhole2D:
    """
    Gaussian q smearing of 2D data (``resolution2d.py:28-115``): each
    measured (qx, qy) is replaced by nr x nphi points of a polar
    oversampling of its resolution ellipse; ``apply`` takes the theory at
    those points (bin-major, ``q_calc = [qx_calc, qy_calc]``) and returns the
    weighted average per measured point.  *data* carries ``qx_data``,
    ``qy_data``, ``q_data`` and optionally ``dqx_data``/``dqy_data``.
    """

    def __init__(self, data=None, index=None, nsigma=NSIGMA_2D, accuracy='Low',
                 coords='polar', device=None):
        self.nr = NR[accuracy.lower()]
        self.nphi = NPHI[accuracy.lower()]
        self.nsigma = nsigma
        self.coords = coords
        self._device_arg = device
        self.index = index if index is not None else slice(None)
        self.qx_data = data.qx_data[self.index]
        self.qy_data = data.qy_data[self.index]
        self.q_data = data.q_data[self.index]
        dqx = getattr(data, 'dqx_data', None)
        dqy = getattr(data, 'dqy_data', None)
        if dqx is not None and dqy is not None:
            self.dqx_data = np.array(dqx[self.index], 'd')
            self.dqy_data = np.array(dqy[self.index], 'd')
            self.dqx_data[self.dqx_data < SIGMA_ZERO] = SIGMA_ZERO
            self.dqy_data[self.dqy_data < SIGMA_ZERO] = SIGMA_ZERO
            qx_calc, qy_calc, weights = self._calc_res()
            self.q_calc = [qx_calc, qy_calc]
            self.q_calc_weights = weights
        else:
            self.dqx_data = self.dqy_data = None
            self.q_calc = [self.qx_data, self.qy_data]
            self.q_calc_weights = None
        self._w_dev = None

    @property
    def device(self):
        return _device(self._device_arg)

    def _calc_res(self):
        """Oversampling points and their gaussian ring weights
        (``resolution2d.py:91-160``), bin-major: point b*nq + i is bin b of
        measured point i."""
        nr, nphi = self.nr, self.nphi
        nbins = nr*nphi
        nq = len(self.qx_data)
        bin_size = self.nsigma/nr
        r = bin_size/2.0 + np.arange(nr)*bin_size
        dphi = (np.arange(nphi)*2.0*np.pi/nphi).repeat(nr).repeat(nq)
        q_phi = np.arctan(self.qy_data/self.qx_data).repeat(nbins).reshape(
            [nq, nbins]).transpose().flatten()
        weight_res = (np.exp(-0.5*(r - bin_size/2.0)**2) - np.exp(-0.5*(r + bin_size/2.0)**2))
        weight_res = weight_res.repeat(nphi).reshape(nr, nphi).transpose().flatten()
        dr = r.repeat(nphi).reshape(nr, nphi).transpose().flatten()
        dqx = np.outer(dr, self.dqx_data).flatten()
        dqy = np.outer(dr, self.dqy_data).flatten()
        qx = self.qx_data.repeat(nbins).reshape(nq, nbins).transpose().flatten()
        qy = self.qy_data.repeat(nbins).reshape(nq, nbins).transpose().flatten()
        if self.coords == 'polar':
            q_r = np.sqrt(qx**2 + qy**2)
            qx_res = ((dqx*np.cos(dphi) + q_r)*np.cos(-q_phi)
                      + dqy*np.sin(dphi)*np.sin(-q_phi))
            qy_res = (-(dqx*np.cos(dphi) + q_r)*np.sin(-q_phi)
                      + dqy*np.sin(dphi)*np.cos(-q_phi))
        else:
            qx_res = qx + dqx*np.cos(dphi)
            qy_res = qy + dqy*np.sin(dphi)
        return qx_res, qy_res, weight_res

    def apply(self, theory, stream=None):
        """Weighted average over the oversampling bins (bins in order, as
        ``np.average(..., axis=0)``); CUDA tensor in -> CUDA tensor out, host
        array in -> host array out."""
        import torch
        if self.q_calc_weights is None:
            return theory
        nq, nbins = len(self.qx_data), self.nr*self.nphi
        on_device = isinstance(theory, torch.Tensor) and theory.is_cuda
        t = (theory if on_device else
             torch.as_tensor(np.ascontiguousarray(theory, 'd'), device=self.device))
        t = t.to(torch.float64).contiguous()
        if t.numel() != nq*nbins:
            raise ValueError("theory has %d points, q_calc %d" % (t.numel(), nq*nbins))
        if self._w_dev is None:
            self._w_dev = torch.as_tensor(np.ascontiguousarray(self.q_calc_weights, 'd'),
                                          device=self.device)
            # the normalisation formed exactly as np.average forms it
            wgt = np.broadcast_to(np.asarray(self.q_calc_weights, 'd'), (1, nbins))
            self._wsum = float(wgt.swapaxes(-1, 0).sum(axis=0)[0])
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(st):
            out = torch.empty(nq, dtype=torch.float64, device=self.device)
            _check(_lib().sasb200_pinhole2d_average(nq, nbins, t.data_ptr(),
                                                    self._w_dev.data_ptr(), self._wsum,
                                                    out.data_ptr(), st.cuda_stream),
                   "pinhole2d_average")
        if on_device:
            return out
        st.synchronize()
        return out.cpu().numpy()


def nllf_sets(theory, Iq, dIq, stream):
    """0.5 sum(((theory - Iq)/dIq)^2) of every row of the CUDA tensor
    *theory* [n_sets, nq] (``bumps_model.py:263-282``), on *stream*; returns
    a CUDA tensor [n_sets]."""
    import torch
    n_sets, nq = theory.shape
    dev = theory.device
    with torch.cuda.device(dev), torch.cuda.stream(stream):
        y = torch.as_tensor(np.ascontiguousarray(Iq, 'd'), device=dev)
        dy = torch.as_tensor(np.ascontiguousarray(dIq, 'd'), device=dev)
        if y.numel() != nq or dy.numel() != nq or theory.stride(1) != 1:
            raise ValueError("data has %d points, theory %d" % (y.numel(), nq))
        out = torch.empty(n_sets, dtype=torch.float64, device=dev)
        _check(_lib().sasb200_nllf_sets(n_sets, nq, theory.data_ptr(), theory.stride(0),
                                        y.data_ptr(), dy.data_ptr(), out.data_ptr(),
                                        stream.cuda_stream), "nllf_sets")
    return out
