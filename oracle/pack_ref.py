"""
CPU restatement of the device packer (csrc/pack.cu) -- test infrastructure
only: tests use it as the checker; the product never imports it.

`expand(ca)` writes the values vector of every set of a column table
(``sasmodels_b200.pack.column_args``) the way ``make_kernel_args``
(sasmodels/details.py:225-254) lays it out, with the gaussian meshes of
``Dispersion._linspace`` / ``GaussianDispersion._weights`` / ``get_weights``
(sasmodels/weights.py:78-102, 264-291): numpy.linspace arithmetic
(i*step + start, the last point = stop), each operation rounded on its own,
the weights' sum in numpy's pairwise order, math.exp for the exponential.

Pinned by tests/test_pack.py against the reference-equivalent host
marshaling (``make_call_args``, itself checked bit for bit against the
reference's own ``make_kernel_args`` in tests/test_host.py).
"""

import math

import numpy as np


def pairwise_sum(a):
    """numpy's add.reduce order for a contiguous float64 row."""
    n = len(a)
    if n < 8:
        res = -0.0
        for v in a:
            res += v
        return res
    if n <= 128:
        r = [float(v) for v in a[:8]]
        i = 8
        while i < n - n % 8:
            for j in range(8):
                r[j] += a[i + j]
            i += 8
        res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]))
        while i < n:
            res += a[i]
            i += 1
        return res
    n2 = n//2
    n2 -= n2 % 8
    return pairwise_sum(a[:n2]) + pairwise_sum(a[n2:])


def gaussian_mesh(value, width, nsigma, npts, relative):
    """(x, normalised w) of one dispersed parameter."""
    sigma = width*value if relative else width
    center = value if relative else 0.0
    lo = (-nsigma)*sigma
    hi = nsigma*sigma
    delta = hi - lo
    div = float(npts - 1)
    step = delta/div
    x = np.empty(npts)
    w = np.empty(npts)
    for i in range(npts):
        y = (i/div)*delta if step == 0.0 else i*step
        y = y + lo
        if i == npts - 1:
            y = hi
        x[i] = center + y
        d = x[i] - center
        w[i] = math.exp((d*d)/((-2.0*sigma)*sigma))
    total = pairwise_sum(w)
    return x, w/total


def expand(ca):
    """The concatenated values vectors of every set of the table `ca`
    (host-marshaled sets copied from ca["host_values"])."""
    scalars, widths, nsigmas = ca["scalars"], ca["widths"], ca["nsigmas"]
    npts, flags, sizes = ca["npts"], ca["flags"], ca["val_sizes"]
    n, nvalues = scalars.shape
    out = []
    for s in range(n):
        if s in ca["host_values"]:
            out.append(np.asarray(ca["host_values"][s], float))
            continue
        xs, ws = [], []
        for k in range(npts.shape[1]):
            value = scalars[s, 2 + k]
            if npts[s, k] <= 0:
                xs.append([value if flags[k] & 2 else 0.0])
                ws.append([1.0])
                continue
            x, w = gaussian_mesh(value, widths[s, k], nsigmas[s, k], int(npts[s, k]),
                                 bool(flags[k] & 1))
            xs.append(x)
            ws.append(w)
        v = np.concatenate([scalars[s]] + [np.asarray(x) for x in xs]
                           + [np.asarray(w) for w in ws])
        out.append(np.concatenate([v, np.zeros(int(sizes[s]) - v.size)]))
    return np.concatenate(out) if out else np.zeros(0)
