"""
Kernel call marshaling: the int32 ``CallDetails`` buffer and the packed
``values`` vector that every kernel entry point reads.

The buffer layouts are a fixed interface shared with the reference DLL
(``sasmodels/kernel_iq.c:47-58`` for ProblemDetails, ``sasmodels/details.py``
for the packing), so the same arrays can be handed to the reference DLL and
to the B200 kernels in the parity tests.
"""

import numpy as np
from numpy import cos, radians, sin

from .modelinfo import NUM_COMMON_PARS, NUM_MAGNETIC_PARS


class CallDetails:
    """
    Polydispersity loop descriptor (``details.py:43-180``).

    ``buffer`` is int32[4*max_pd + 4]::

        pd_par[max_pd]     kernel-parameter index of each pd dimension
        pd_length[max_pd]  number of points in each dimension
        pd_offset[max_pd]  offset of its values/weights in the pd block
        pd_stride[max_pd]  mixed-radix stride (cumulative product of lengths)
        num_eval           total mesh size
        num_weights        total length of the pd value (and weight) block
        num_active         number of dimensions with length > 1
        theta_par          kernel-parameter index of theta, or -1
    """
    def __init__(self, model_info):
        parameters = model_info.parameters
        max_pd = parameters.max_pd
        self.max_pd = max_pd
        self.buffer = np.zeros(4*max_pd + 4, 'i4')
        self.theta_par = parameters.theta_offset
        self.offset = None
        self.length = None
        self.info = model_info

    def _view(self, k):
        return self.buffer[k*self.max_pd:(k+1)*self.max_pd]

    pd_par = property(lambda self: self._view(0))
    pd_length = property(lambda self: self._view(1))
    pd_offset = property(lambda self: self._view(2))
    pd_stride = property(lambda self: self._view(3))

    def _get(k):
        return property(lambda self: int(self.buffer[k]),
                        lambda self, v: self.buffer.__setitem__(k, v))
    num_eval = _get(-4)
    num_weights = _get(-3)
    num_active = _get(-2)
    theta_par = _get(-1)
    del _get


def make_details(model_info, length, offset, num_weights):
    """
    Sort the pd dimensions by decreasing length and set the strides so that
    dimension 0 (the longest) varies fastest (``details.py:183-221``).
    """
    num_active = int(np.sum(length > 1))
    max_pd = model_info.parameters.max_pd
    if num_active > max_pd:
        raise ValueError("Too many polydisperse parameters")
    idx = np.argsort(length)[::-1][:max_pd]
    pd_stride = np.cumprod(np.hstack((1, length[idx])))

    call_details = CallDetails(model_info)
    call_details.pd_par[:max_pd] = idx
    call_details.pd_length[:max_pd] = length[idx]
    call_details.pd_offset[:max_pd] = offset[idx]
    call_details.pd_stride[:max_pd] = pd_stride[:-1]
    call_details.num_eval = int(pd_stride[-1])
    call_details.num_weights = int(num_weights)
    call_details.num_active = num_active
    call_details.length = length
    call_details.offset = offset
    return call_details


_ZEROS = tuple([0.]*31)


def make_kernel_args(kernel, mesh):
    """
    Pack ``[scale, background, pars..., (magnetic block)]`` followed by all pd
    values then all pd weights, zero padded to a multiple of 32 entries
    (``details.py:225-254``).  Returns (call_details, values, is_magnetic).
    """
    info = kernel.info
    npars = info.parameters.npars
    nvalues = info.parameters.nvalues
    scalars = [value for value, _dispersity, _weight in mesh]
    if npars:
        _, dispersity, weight = zip(*mesh[NUM_COMMON_PARS:npars+NUM_COMMON_PARS])
    else:
        dispersity, weight = (), ()
    length = np.array([len(w) for w in weight])
    offset = np.cumsum(np.hstack((0, length)))
    call_details = make_details(info, length, offset[:-1], offset[-1])
    data_len = nvalues + 2*sum(len(v) for v in dispersity)
    extra = (32 - data_len % 32) % 32
    data = np.hstack((scalars,) + tuple(dispersity) + tuple(weight) + _ZEROS[:extra])
    data = data.astype(np.dtype(getattr(kernel, 'dtype', 'd')))
    is_magnetic = convert_magnetism(info.parameters, data)
    return call_details, data, is_magnetic


def convert_magnetism(parameters, values):
    """
    In place (M0, mtheta, mphi) -> (mx, my, mz) for every sld; True if any
    M0 is non-zero (``details.py:288-306``).
    """
    nmagpars = NUM_MAGNETIC_PARS*parameters.nmagnetic
    if nmagpars == 0:
        return False
    mag = values[parameters.nvalues-nmagpars:parameters.nvalues]
    mag = mag.reshape(-1, NUM_MAGNETIC_PARS)
    if np.any(mag[:, 0] != 0.0):
        M0 = mag[:, 0].copy()
        theta, phi = radians(mag[:, 1]), radians(mag[:, 2])
        mag[:, 0] = M0*sin(theta)*cos(phi)
        mag[:, 1] = M0*sin(theta)*sin(phi)
        mag[:, 2] = M0*cos(theta)
        return True
    return False


def validate_call(info, details, values):
    """
    Check that a details buffer and values vector are consistent with each
    other and with *info* before they reach the device: every mesh index the
    kernels can form from them must land inside *values*.  Raises ValueError.
    """
    table = info.parameters
    max_pd = table.max_pd
    buf = np.asarray(details, np.int64)
    if buf.size != 4*max_pd + 4:
        raise ValueError("details has %d entries, expected %d" % (buf.size, 4*max_pd + 4))
    pd_par, pd_length = buf[:max_pd], buf[max_pd:2*max_pd]
    pd_offset, pd_stride = buf[2*max_pd:3*max_pd], buf[3*max_pd:4*max_pd]
    num_eval, num_weights = int(buf[4*max_pd]), int(buf[4*max_pd + 1])
    if num_weights < 0 or len(values) < table.nvalues + 2*num_weights:
        raise ValueError("values vector too short for %d dispersity weights" % num_weights)
    expected = 1
    for d in range(max_pd):
        if not 0 <= pd_par[d] < max(table.npars, 1):
            raise ValueError("pd_par[%d] = %d out of range" % (d, pd_par[d]))
        if pd_length[d] < 0 or pd_offset[d] < 0 \
                or pd_offset[d] + pd_length[d] > num_weights:
            raise ValueError("pd dimension %d outside the weight vector" % d)
        if pd_stride[d] != expected:
            raise ValueError("pd_stride[%d] = %d, expected %d" % (d, pd_stride[d], expected))
        expected *= int(pd_length[d])
    if num_eval != expected or num_eval >= 2**31:
        raise ValueError("num_eval = %d does not match the pd lengths (%d)"
                         % (num_eval, expected))
