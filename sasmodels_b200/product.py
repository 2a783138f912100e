"""
P@S products (form factor times structure factor) with the whole chain on
the device.

Mirrors ``sasmodels/product.py``: :func:`make_product_info` builds the
combined parameter table the same way (``product.py:171-234``: P's
parameters, then S's with S.volfraction dropped when P has one and clashing
names tagged ``_S``, then ``structure_factor_mode`` and
``radius_effective_mode``, then P's magnetic block), so a product is
marshaled by the ordinary ``make_call_args``; :class:`B200ProductKernel`
splits the call the way ``ProductKernel.Iq`` does (``product.py:430-553``).

The difference is where it runs.  The reference calls P.Fq, copies <F>,
<F^2>, R_eff and the volume ratio to the host, patches S's values vector
there, calls S.Iq and combines on the host.  Here P's sums stay on the
device: R_eff and volfraction x V_form/V_shell are written into S's values
vector on the device, S runs on the same stream, and the combination
scale/V (<F^2> + <F>^2 (S - 1)) + background (beta approximation) or
scale/V <F^2> S + background is formed there too; only the final I(q)
crosses to the host.
"""

import copy

import numpy as np

from .details import make_details
from .modelinfo import NUM_COMMON_PARS, ModelInfo, Parameter

STRUCTURE_MODE_ID = "structure_factor_mode"
RADIUS_MODE_ID = "radius_effective_mode"
RADIUS_ID = "radius_effective"
VOLFRAC_ID = "volfraction"


def _tag(par):
    par = copy.copy(par)
    par.id = par.name = par.name + "_S"
    return par


def make_product_info(p_info, s_info):
    """Combined model info of P@S (``product.py:171-234``)."""
    sk = s_info.parameters.kernel_parameters
    if not len(sk) >= 2:
        raise TypeError("S needs %s and %s as its first parameters" % (RADIUS_ID, VOLFRAC_ID))
    if sk[0].id != RADIUS_ID:
        raise TypeError("S needs %s as first parameter" % RADIUS_ID)
    if sk[1].id != VOLFRAC_ID:
        raise TypeError("S needs %s as second parameter" % VOLFRAC_ID)
    if s_info.parameters.nmagnetic:
        raise TypeError("S should not have SLD parameters")
    if RADIUS_ID in p_info.parameters:
        raise TypeError("P should not have %s" % RADIUS_ID)
    pt, st = p_info.parameters, s_info.parameters
    p_has_volfrac = VOLFRAC_ID in pt
    p_set = set(p.id for p in pt.kernel_parameters)

    def s_part(pars):
        return [(_tag(p) if p.id in p_set else p) for p in pars
                if p.id != VOLFRAC_ID or not p_has_volfrac]

    s_kernel = s_part(sk)
    s_call = s_part(st.call_parameters[NUM_COMMON_PARS:NUM_COMMON_PARS + st.npars])
    extras = []
    if p_info.have_Fq:
        extras.append(Parameter(STRUCTURE_MODE_ID, "", 0, (0.0, 1.0), "",
                                "Structure factor calculation"))
    if p_info.radius_effective_modes:
        n = len(p_info.radius_effective_modes)
        extras.append(Parameter(RADIUS_MODE_ID, "", 1, (0.0, float(n)), "",
                                "Effective radius calculation"))
    p_call = pt.call_parameters
    kernel = list(pt.kernel_parameters) + s_kernel + extras
    call = (p_call[:NUM_COMMON_PARS + pt.npars] + s_call + extras
            + p_call[NUM_COMMON_PARS + pt.npars:])
    d = dict(p_info.raw)
    d.update(id="@".join((p_info.id, s_info.id)), name="@".join((p_info.name, s_info.name)),
             have_Fq=False, radius_effective_modes=[], structure_factor=False,
             npars=pt.npars + len(s_call) + len(extras), nmagnetic=pt.nmagnetic,
             max_pd=pt.max_pd + st.max_pd,
             kernel_parameters=[p.as_dict() for p in kernel],
             call_parameters=[p.as_dict() for p in call])
    info = ModelInfo(d)
    info.raw["nvalues"] = info.parameters.nvalues
    info.composition = ("product", [p_info, s_info])
    return info


class B200ProductModel:
    """Engine for a P@S model: a B200 model for P and one for S."""

    def __init__(self, model_info, P, S):
        self.info = model_info
        self.P = P
        self.S = S
        self.dtype = P.dtype

    def make_kernel(self, q_vectors):
        return B200ProductKernel(self.info, self.P.make_kernel(q_vectors),
                                 self.S.make_kernel(q_vectors), q_vectors)

    def release(self):
        pass


class B200ProductKernel:
    """``ProductKernel`` (``product.py:364-560``) with P, the patching of S's
    values and the combination on the device."""

    def __init__(self, model_info, p_kernel, s_kernel, q):
        self.info = model_info
        self.q = q
        self.p_kernel = p_kernel
        self.s_kernel = s_kernel
        self.dtype = p_kernel.dtype
        self.dim = p_kernel.dim
        self.q_input = p_kernel.q_input
        self.results = None
        table = model_info.parameters
        for k, p in enumerate(table.call_parameters):
            if p.id == VOLFRAC_ID:
                self._volfrac_index = k
                break
        else:
            raise RuntimeError("no %s parameter in %s" % (VOLFRAC_ID, self))
        p_info, s_info = model_info.composition[1]
        p_npars = p_info.parameters.npars
        s_npars = s_info.parameters.npars
        have_beta_mode = p_info.have_Fq
        have_er_mode = bool(p_info.radius_effective_modes)
        volfrac_in_p = self._volfrac_index < p_npars + NUM_COMMON_PARS
        self._p_detail_slice = slice(0, p_npars)
        self._s_detail_slice = slice(p_npars, p_npars + s_npars - volfrac_in_p)
        self._volfrac_in_p = volfrac_in_p
        first_p, last_p = NUM_COMMON_PARS, p_npars + NUM_COMMON_PARS
        self._p_value_slice = slice(first_p, last_p)
        self._er_index = last_p
        first_s = last_p + NUM_COMMON_PARS - volfrac_in_p
        last_s = first_s + s_npars - NUM_COMMON_PARS
        self._s_value_slice = slice(first_s, last_s)
        self._s_dist_start = NUM_COMMON_PARS + s_npars
        self._beta_mode_index = last_s if have_beta_mode else 0
        self._er_mode_index = last_s + have_beta_mode if have_er_mode else 0
        first_mag = last_s + have_beta_mode + have_er_mode
        mag_pars = 3*p_info.parameters.nmagnetic
        last_mag = first_mag + (mag_pars + 4 if mag_pars else 0)
        self._magnetic_slice = slice(first_mag, last_mag)

    def Iq(self, call_details, values, cutoff, magnetic):
        import torch
        p_info, s_info = self.info.composition[1]
        pk, sk = self.p_kernel, self.s_kernel
        scale, background = values[0], values[1]
        volfrac = values[self._volfrac_index]
        er_mode = int(values[self._er_mode_index]) if self._er_mode_index > 0 else 0
        beta_mode = values[self._beta_mode_index] > 0 if self._beta_mode_index > 0 else False
        nvalues = self.info.parameters.nvalues
        nweights = call_details.num_weights
        weights = values[nvalues:nvalues + 2*nweights]
        if beta_mode and pk.dim == '2d':
            raise NotImplementedError("beta not yet supported for 2D")

        # P: values as the reference builds them (product.py:461-471)
        p_length = call_details.length[self._p_detail_slice]
        p_offset = call_details.offset[self._p_detail_slice]
        p_details = make_details(p_info, p_length, p_offset, nweights)
        p_values = [[1., 0.], values[self._p_value_slice], values[self._magnetic_slice],
                    weights]
        spacer = (32 - sum(len(v) for v in p_values) % 32) % 32
        p_values.append([0.]*spacer)
        p_values = np.hstack(p_values).astype('d')

        # S: values with placeholders for R_eff and volfraction
        # (product.py:480-514); the placeholders are filled on the device
        s_length = call_details.length[self._s_detail_slice]
        s_offset = call_details.offset[self._s_detail_slice]
        if self._volfrac_in_p:
            s_length = np.insert(s_length, 1, 1)
            s_offset = np.insert(s_offset, 1, p_offset[self._volfrac_index - 2])
        if er_mode > 0:
            s_length[0] = 1
        s_details = make_details(s_info, s_length, s_offset, nweights)
        s_values = [[1., 0., values[self._er_index], 0.], values[self._s_value_slice], weights]
        spacer = (32 - sum(len(v) for v in s_values) % 32) % 32
        s_values.append([0.]*spacer)
        s_values = np.hstack(s_values).astype('d')
        d0 = self._s_dist_start
        if er_mode > 0:
            s_values[d0 + s_offset[0] + nweights] = 1.0
        s_values[d0 + s_offset[1] + nweights] = 1.0

        nq = pk.q_input.nq
        stream = pk.stream
        dd_p, dv_p = pk.upload(p_details, p_values)
        with torch.cuda.device(pk.device), torch.cuda.stream(stream):
            # a nonzero mode also makes the library sum the volumes (and R_eff)
            # in the DLL's own mesh order, so the S inputs below equal the
            # reference's bit for bit; with er_mode 0 the R_eff slot is unused
            res = pk.launch(pk.variant(magnetic), dd_p, dv_p, 0, p_details.num_eval, cutoff,
                            er_mode if er_mode > 0 else 1)
            nout = 2 if p_info.have_Fq and pk.dim == '1d' else 1
            tail = res[nout*nq:nout*nq + 4]
            total = torch.where(tail[0] == 0, torch.ones_like(tail[0]), tail[0])
            form = tail[1]/total
            shell = tail[2]/total
            reff = tail[3]/total
            shell = torch.where(shell == 0, torch.ones_like(shell), shell)
            F2 = res[0:nout*nq:nout]/total
            F1 = res[1:nout*nq:nout]/total if nout == 2 else None
            ratio = form/shell
        # S on the same stream, its values patched on the device
        sk.stream.wait_stream(stream)
        dd_s, dv_s = sk.upload(s_details, s_values)
        with torch.cuda.device(sk.device), torch.cuda.stream(sk.stream):
            vf = volfrac*ratio
            dv_s[NUM_COMMON_PARS + 1] = vf
            dv_s[d0 + int(s_offset[1])] = vf
            if er_mode > 0:
                dv_s[NUM_COMMON_PARS] = reff
                dv_s[d0 + int(s_offset[0])] = reff
            sres = sk.launch(sk.variant(False), dd_s, dv_s, 0, s_details.num_eval, cutoff, 0)
            s_nout = 2 if s_info.have_Fq and sk.dim == '1d' else 1
            st = sres[s_nout*nq:s_nout*nq + 4]
            s_total = torch.where(st[0] == 0, torch.ones_like(st[0]), st[0])
            s_shell = st[2]/s_total
            s_shell = torch.where(s_shell == 0, torch.ones_like(s_shell), s_shell)
            S = (1.0/s_shell)*(sres[0:s_nout*nq:s_nout]/s_total) + 0.0
            PS = F2 + F1**2*(S - 1) if beta_mode else F2*S
            combined = scale/shell
            if not self._volfrac_in_p:
                combined = combined*volfrac
            I = combined*PS + background
            if pk.q_input.order_dev is not None:
                I = torch.empty_like(I).index_copy_(0, pk.q_input.order_dev, I)
            out = I.cpu().numpy()
        self.results = dict(F=F1, Fsq=F2, S=S, radius_effective=reff, shell_volume=shell,
                            volume_ratio=ratio, beta_mode=beta_mode)
        return out

    __call__ = Iq

    def release(self):
        self.p_kernel.release()
        self.s_kernel.release()
