"""
CPU restatement of the device packer (csrc/pack.cu) -- test infrastructure
only: tests use it as the checker; the product never imports it.

`expand(ca)` writes the values vector of every set of a column table
(``sasmodels_b200.pack.column_args``) the way ``make_kernel_args``
(sasmodels/details.py:225-254) lays it out, with the dispersity meshes of
every distribution of sasmodels/weights.py (:21-220, 264-291) --
numpy.linspace arithmetic (i*step + start, the last point = stop) over the
kept index range, each operation rounded on its own, the weights' sum in
numpy's pairwise order, math.exp/log/lgamma for the densities -- and the
magnetic conversion of details.py:288-306 (math.sin/cos).

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


KINDS = ("gaussian", "uniform", "rectangle", "lognormal", "schulz", "boltzmann")
DEG = 0.017453292519943295        # numpy.radians factor pi/180


def density(kind, x, c, sigma):
    """Unnormalised density of the distributions of sasmodels/weights.py
    (:86-220) at x, each operation rounded on its own."""
    if kind == "gaussian":
        d = x - c
        return math.exp((d*d)/((-2.0*sigma)*sigma))
    if kind == "lognormal":
        s = math.fabs(sigma/c)
        t = (math.log(x) - math.log(c))/s
        return math.exp(-0.5*(t*t))/(x*s)
    if kind == "schulz":
        R = x/c
        q = c/sigma
        z = q*q
        a = z*math.log(z) + (z - 1.0)*math.log(R) - R*z - math.log(c) - math.lgamma(z)
        return math.exp(a)
    if kind == "boltzmann":
        return math.exp(-math.fabs(x - c)/math.fabs(sigma))
    return 1.0      # uniform, rectangle


def mesh(kind, value, width, nsigma, ntot, first, npts, relative):
    """(x, normalised w) of one dispersed parameter: points first ..
    first + npts - 1 of the distribution's ntot-point numpy.linspace."""
    sigma = width*value if relative else width
    center = value if relative else 0.0
    flat = kind == "uniform"
    lo = center - sigma if flat else (-nsigma)*sigma
    hi = center + sigma if flat else nsigma*sigma
    delta = hi - lo
    div = float(ntot - 1)
    step = delta/div
    x = np.empty(npts)
    w = np.empty(npts)
    for j in range(npts):
        i = first + j
        y = (i/div)*delta if step == 0.0 else i*step
        y = y + lo
        if i == ntot - 1:
            y = hi
        x[j] = y if flat else center + y
        w[j] = density(kind, x[j], center, sigma)
    total = pairwise_sum(w)
    return x, w/total


def gaussian_mesh(value, width, nsigma, npts, relative):
    """(x, normalised w) of an unclipped gaussian."""
    return mesh("gaussian", value, width, nsigma, npts, 0, npts, relative)


def convert_magnetism(scalars, nmag):
    """(M0, mtheta, mphi) -> (mx, my, mz) of the last nmag triples
    (details.py:288-306), in place."""
    nvalues = len(scalars)
    for m in range(nmag):
        k = nvalues - 3*nmag + 3*m
        M0, th, ph = scalars[k], scalars[k + 1]*DEG, scalars[k + 2]*DEG
        Ms = M0*math.sin(th)
        scalars[k], scalars[k + 1], scalars[k + 2] = Ms*math.cos(ph), Ms*math.sin(ph), \
            M0*math.cos(th)


def expand(ca):
    """The concatenated values vectors of every set of the table `ca`
    (host-marshaled sets copied from ca["host_values"])."""
    scalars, widths, nsigmas = ca["scalars"], ca["widths"], ca["nsigmas"]
    npts, flags, sizes = ca["npts"], ca["flags"], ca["val_sizes"]
    first, ntot, kinds = ca["first"], ca["ntot"], ca["kinds"]
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
            x, w = mesh(KINDS[kinds[s, k]], value, widths[s, k], nsigmas[s, k],
                        int(ntot[s, k]), int(first[s, k]), int(npts[s, k]),
                        bool(flags[k] & 1))
            xs.append(x)
            ws.append(w)
        head = scalars[s].copy()
        if ca["magnetic"][s]:
            convert_magnetism(head, int(ca["nmag"]))
        v = np.concatenate([head] + [np.asarray(x) for x in xs]
                           + [np.asarray(w) for w in ws])
        out.append(np.concatenate([v, np.zeros(int(sizes[s]) - v.size)]))
    return np.concatenate(out) if out else np.zeros(0)
