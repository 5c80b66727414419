"""Plan: one horizontal resolution (l_max, minc) resident on one GPU.

A Plan owns the FP64 Legendre tables (built on the device by
``mt_plan_create``) and exposes the transforms and nonlinear-term builders
on torch CUDA tensors.  Shapes, dtypes and conventions are those of the
reference's ``magic_torch.sht`` (spectral (lm_max,) / (lm_max, B) complex128,
grids (n_theta, n_phi) / (B, n_theta, n_phi) float64 with interleaved N/S
theta rows).  Every call enqueues on the current torch CUDA stream and does not
synchronise the host.
"""

import collections
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import MagicError, check, raise_device_status

_CD = torch.complex128
_RD = torch.float64


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


class _StatusWatch:
    """Non-blocking check of the split kernels' device status.  After each call
    the status word of its workspace (first int, written by a bounded tensor-pipe
    wait that ran out) is copied on the same stream into a pinned host slot, and
    an event marks when it has landed; poll() raises MagicError for the first
    landed non-zero code.  Nothing is recorded while the stream is being captured
    into a CUDA graph (the caller reads the word after replays instead)."""

    SLOTS = 4096

    def __init__(self):
        self.host = torch.zeros(self.SLOTS, dtype=torch.int32).pin_memory()
        self.pending = collections.deque()
        self.next = 0

    def record(self, work, what):
        if torch.cuda.is_current_stream_capturing():
            return
        self.poll()
        if len(self.pending) >= self.SLOTS:
            self.poll(block=True)
        stream = torch.cuda.current_stream(work.device)
        slot = self.next
        self.next = (self.next + 1) % self.SLOTS
        self.host[slot:slot + 1].copy_(work[:4].view(torch.int32), non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        self.pending.append((slot, ev, what))

    def poll(self, block=False):
        while self.pending:
            slot, ev, what = self.pending[0]
            if block:
                ev.synchronize()
            elif not ev.query():
                return
            self.pending.popleft()
            code = int(self.host[slot])
            if code:
                self.pending.clear()
                raise_device_status(code, what)


class Plan:
    """Tables and entry points for one (l_max, minc) grid on one CUDA device.

    Split-precision plans watch the device status of every call (see
    ``poll_status``): a bounded wait on the tensor pipe that ran out is raised
    as MagicError by the next call on the plan, or by ``poll_status``."""

    def __init__(self, l_max, minc=1, precision="fp64", device=None, n_theta_max=0,
                 n_phi_max=0):
        if not torch.cuda.is_available():
            raise RuntimeError("magic_b200 needs a CUDA device (B200); no CPU fallback")
        dev = torch.device(device if device is not None else "cuda")
        if dev.type != "cuda":
            raise ValueError("magic_b200 plans live on CUDA devices")
        self.device = dev if dev.index is not None else torch.device(
            "cuda", torch.cuda.current_device())
        prec = {"fp64": _lib.MT_PREC_FP64, "split": _lib.MT_PREC_SPLIT,
                "ozaki": _lib.MT_PREC_OZAKI}[precision]
        self.precision = precision
        L = _lib.lib()
        desc = _lib.GridDesc(int(l_max), int(minc), int(n_theta_max), int(n_phi_max), prec)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(L.mt_plan_create(C.byref(desc), C.byref(h)))
        self._h = h
        info = _lib.PlanInfo()
        check(L.mt_plan_get_info(h, C.byref(info)))
        self.l_max = info.l_max
        self.minc = info.minc
        self.n_theta_max = info.n_theta_max
        self.n_phi_max = info.n_phi_max
        self.n_m_max = info.n_m_max
        self.lm_max = info.lm_max
        self.nhs = info.nhs
        ls, l_of, m_of = [], [], []
        pos = 0
        for m in range(0, self.l_max + 1, self.minc):
            ls.append(pos)
            for l in range(m, self.l_max + 1):
                l_of.append(l)
                m_of.append(m)
            pos += self.l_max - m + 1
        self.lStart = np.array(ls)
        self.lm2l = np.array(l_of)
        self.lm2m = np.array(m_of)
        lf = torch.tensor(self.lm2l, dtype=_RD, device=self.device)
        self.dLh = lf * (lf + 1.0)
        self.dPhi = 1j * torch.tensor(self.lm2m, dtype=_RD, device=self.device).to(_CD)
        th = torch.empty(self.n_theta_max, dtype=_RD, device=self.device)
        check(L.mt_plan_copy_tables(h, _ptr(th), None, None, None, self._stream()))
        gi = torch.zeros(self.n_theta_max, dtype=torch.long)
        gi[0::2] = torch.arange(self.nhs)
        gi[1::2] = torch.arange(self.n_theta_max - 1, self.nhs - 1, -1)
        self.grid_idx = gi.to(self.device)
        sin_g = torch.sin(th[self.grid_idx])
        self.O_sin_theta_E2_grid = 1.0 / sin_g ** 2
        self._status = _StatusWatch() if precision != "fp64" else None

    # ------------------------------------------------------ device status
    def poll_status(self, block=False):
        """Raise MagicError if a split-precision call on this plan recorded a
        device-side timeout.  block=False only looks at calls that have already
        finished; block=True waits for every call made so far."""
        if self._status is not None:
            self._status.poll(block)

    def device_status(self, work):
        """Status word of the call that last used ``work`` (synchronises the
        current stream): 0, or the code of the bounded wait that ran out."""
        code = C.c_int(0)
        check(_lib.lib().mt_device_status(_ptr(work), C.byref(code), self._stream()))
        return code.value

    def _watch(self, work, what, fused=False):
        """Record the status word of a call that cleared it: every call of a split
        plan; on digit-split (ozaki) plans only the fused stage (their transforms
        run the FP64 kernels, which leave the word alone)."""
        if self._status is not None and (fused or self.precision == "split"):
            self._status.record(work, what)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().mt_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------ helpers
    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _work(self, nbytes):
        return torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=self.device)

    def _spec2d(self, x, name):
        if not isinstance(x, torch.Tensor) or x.device != self.device:
            raise ValueError(f"{name}: expected a tensor on {self.device}")
        one = x.dim() == 1
        x2 = x.unsqueeze(1) if one else x
        if x2.dim() != 2 or x2.shape[0] != self.lm_max:
            raise ValueError(f"{name}: expected shape (lm_max={self.lm_max},[B])")
        if x2.dtype != _CD:
            x2 = x2.to(_CD)
        if x2.stride(1) != 1 or x2.stride(0) < x2.shape[1]:
            x2 = x2.contiguous()
        return x2, one

    def _grid3d(self, x, name):
        if not isinstance(x, torch.Tensor) or x.device != self.device:
            raise ValueError(f"{name}: expected a tensor on {self.device}")
        one = x.dim() == 2
        x3 = x.unsqueeze(0) if one else x
        if x3.dim() != 3 or tuple(x3.shape[1:]) != (self.n_theta_max, self.n_phi_max):
            raise ValueError(f"{name}: expected shape ([B,] {self.n_theta_max}, {self.n_phi_max})")
        return x3.to(_RD).contiguous(), one

    def tables(self):
        """FP64 tables built on the device: theta_ord, gauss, Plm, dPlm (reference layout)."""
        nt, lm, nhs = self.n_theta_max, self.lm_max, self.nhs
        out = dict(theta_ord=torch.empty(nt, dtype=_RD, device=self.device),
                   gauss=torch.empty(nt, dtype=_RD, device=self.device),
                   Plm=torch.empty(lm, nhs, dtype=_RD, device=self.device),
                   dPlm=torch.empty(lm, nhs, dtype=_RD, device=self.device))
        check(_lib.lib().mt_plan_copy_tables(self._h, _ptr(out["theta_ord"]), _ptr(out["gauss"]),
                                             _ptr(out["Plm"]), _ptr(out["dPlm"]), self._stream()))
        return out

    # -------------------------------------------------------- transforms
    def scal_to_spat(self, Slm, lcut=None):
        X, one = self._spec2d(Slm, "Slm")
        B = X.shape[1]
        out = torch.empty(B, self.n_theta_max, self.n_phi_max, dtype=_RD, device=self.device)
        L = _lib.lib()
        ws = self._work(L.mt_transform_workspace(self._h, B, 1))
        check(L.mt_scal_to_spat(self._h, _ptr(X), X.stride(0), B, _ptr(out), _ptr(ws),
                                ws.numel(), self._stream()))
        self._watch(ws, "scal_to_spat")
        return out[0] if one else out

    def scal_to_SH(self, sc, lcut=None):
        g, one = self._grid3d(sc, "sc")
        B = g.shape[0]
        out = torch.empty(self.lm_max, B, dtype=_CD, device=self.device)
        L = _lib.lib()
        ws = self._work(L.mt_transform_workspace(self._h, B, 1))
        check(L.mt_scal_to_SH(self._h, _ptr(g), B, _ptr(out), B, _ptr(ws), ws.numel(),
                              self._stream()))
        self._watch(ws, "scal_to_SH")
        return out[:, 0] if one else out

    def torpol_to_spat(self, Qlm, Slm, Tlm, lcut=None):
        Q, one = self._spec2d(Qlm, "Qlm")
        S, _ = self._spec2d(Slm, "Slm")
        T, _ = self._spec2d(Tlm, "Tlm")
        if not (Q.shape == S.shape == T.shape):
            raise ValueError("Qlm, Slm, Tlm must have the same shape")
        if not (Q.stride(0) == S.stride(0) == T.stride(0)):
            Q, S, T = Q.contiguous(), S.contiguous(), T.contiguous()
        B = Q.shape[1]
        outs = [torch.empty(B, self.n_theta_max, self.n_phi_max, dtype=_RD, device=self.device)
                for _ in range(3)]
        L = _lib.lib()
        ws = self._work(L.mt_transform_workspace(self._h, B, 3))
        check(L.mt_torpol_to_spat(self._h, _ptr(Q), _ptr(S), _ptr(T), Q.stride(0), B,
                                  *[_ptr(o) for o in outs], _ptr(ws), ws.numel(), self._stream()))
        self._watch(ws, "torpol_to_spat")
        return tuple(o[0] for o in outs) if one else tuple(outs)

    def spat_to_sphertor(self, vt, vp, lcut=None):
        gt, one = self._grid3d(vt, "vt")
        gp, _ = self._grid3d(vp, "vp")
        if gt.shape != gp.shape:
            raise ValueError("vt and vp must have the same shape")
        B = gt.shape[0]
        S = torch.empty(self.lm_max, B, dtype=_CD, device=self.device)
        T = torch.empty_like(S)
        L = _lib.lib()
        ws = self._work(L.mt_transform_workspace(self._h, B, 2))
        check(L.mt_spat_to_sphertor(self._h, _ptr(gt), _ptr(gp), B, _ptr(S), _ptr(T), B,
                                    _ptr(ws), ws.numel(), self._stream()))
        self._watch(ws, "spat_to_sphertor")
        return (S[:, 0], T[:, 0]) if one else (S, T)

    def _grad(self, Slm, scale_dlh):
        X, one = self._spec2d(Slm, "Slm")
        B = X.shape[1]
        gt = torch.empty(B, self.n_theta_max, self.n_phi_max, dtype=_RD, device=self.device)
        gp = torch.empty_like(gt)
        L = _lib.lib()
        ws = self._work(L.mt_transform_workspace(self._h, B, 2))
        check(L.mt_scal_to_grad_spat(self._h, _ptr(X), X.stride(0), B, int(scale_dlh), _ptr(gt),
                                     _ptr(gp), _ptr(ws), ws.numel(), self._stream()))
        self._watch(ws, "scal_to_grad_spat")
        return (gt[0], gp[0]) if one else (gt, gp)

    def scal_to_grad_spat(self, Slm, lcut=None):
        return self._grad(Slm, False)

    def pol_to_grad_spat(self, Slm, lcut=None):
        return self._grad(Slm, True)

    # ------------------------------------------------- grid-space products
    def _grids(self, arrs, n_r, name):
        out = []
        for i, a in enumerate(arrs):
            if a.shape != (n_r, self.n_theta_max, self.n_phi_max) or a.device != self.device:
                raise ValueError(f"{name}[{i}]: expected ({n_r}, {self.n_theta_max}, "
                                 f"{self.n_phi_max}) on {self.device}")
            out.append(a.to(_RD).contiguous())
        return out

    def _prof(self, x, n_r):
        t = torch.as_tensor(x, dtype=_RD, device=self.device).reshape(-1)
        if t.numel() == 1 and n_r > 1:
            t = t.expand(n_r)
        return t.contiguous()

    def get_nl(self, grids, or2, or4, LFfac):
        """get_nl products (magic_torch/get_nl.py:30-87); grids: 14 (n_r, nt, np)."""
        n_r = grids[0].shape[0]
        ins = self._grids(grids, n_r, "get_nl")
        outs = [torch.empty_like(ins[0]) for _ in range(12)]
        or2 = self._prof(or2, n_r)
        or4 = self._prof(or4, n_r)
        pin = (C.c_void_p * 14)(*[t.data_ptr() for t in ins])
        pout = (C.c_void_p * 12)(*[t.data_ptr() for t in outs])
        check(_lib.lib().mt_get_nl(self._h, n_r, pin, pout, _ptr(or2), _ptr(or4), float(LFfac),
                                   self._stream()))
        return tuple(outs)

    def get_nl_anel(self, grids, prof, LFfac, ViscHeatFac, OhmLossFac, l_mag=True):
        """get_nl_anel products (magic_torch/get_nl_anel.py:41-136); 19 grids in, 13 out.

        ``prof``: dict of radial profiles r, or1, or2, or4, beta, orho1, otemp1, visc,
        lambda_ over the grid levels.
        """
        n_r = grids[0].shape[0]
        ins = self._grids(grids, n_r, "get_nl_anel")
        outs = [torch.empty_like(ins[0]) for _ in range(13)]
        keep = {k: self._prof(prof[k], n_r) for k in
                ("r", "or1", "or2", "or4", "beta", "orho1", "otemp1", "visc", "lambda_")}
        p = _lib.AnelParams(*[k.data_ptr() for k in keep.values()], float(LFfac),
                            float(ViscHeatFac), float(OhmLossFac), int(bool(l_mag)))
        pin = (C.c_void_p * 19)(*[t.data_ptr() for t in ins])
        pout = (C.c_void_p * 13)(*[t.data_ptr() for t in outs])
        check(_lib.lib().mt_get_nl_anel(self._h, n_r, pin, pout, C.byref(p), self._stream()))
        return tuple(outs)

    def courant(self, vr, vt, vp, br, bt, bp, prof, courfac, alffac, LFfac, opm, damp=True):
        """Per-level (dtrkc, dthkc) (magic_torch/courant.py:80-127)."""
        n_r = vr.shape[0]
        mag = br is not None
        g = self._grids([vr, vt, vp] + ([br, bt, bp] if mag else []), n_r, "courant")
        keep = {k: self._prof(prof[k], n_r) for k in
                ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2")}
        mode = (1 if damp else 2) if mag else 0
        p = _lib.CourantParams(*[k.data_ptr() for k in keep.values()], float(courfac),
                               float(alffac), float(LFfac), float(opm), mode)
        dtr = torch.empty(n_r, dtype=_RD, device=self.device)
        dth = torch.empty_like(dtr)
        L = _lib.lib()
        ws = self._work(L.mt_courant_workspace(self._h, n_r))
        bptr = [_ptr(x) for x in g[3:6]] if mag else [C.c_void_p(0)] * 3
        check(L.mt_courant(self._h, n_r, _ptr(g[0]), _ptr(g[1]), _ptr(g[2]), *bptr, C.byref(p),
                           _ptr(dtr), _ptr(dth), _ptr(ws), ws.numel(), self._stream()))
        return dtr, dth

    # --------------------------------------------------- fused stage
    def nl_bouss_workspace(self, n_r, l_mag=True, l_chem=False):
        return _lib.lib().mt_nl_bouss_workspace(self._h, int(n_r), int(l_mag), int(l_chem))

    def nl_bouss(self, fields, prof, LFfac, courfac, alffac, opm, l_mag=True, l_chem=False,
                 damp=True, out=None, work=None, parts=0, LFfac_r=None):
        """Fused Boussinesq nonlinear stage (magic_torch/step_time.py:931-1213, steps 1-3 + CFL).

        ``fields``: dict of spectral (lm_max, n_r) complex128 arrays w, dw, ddw, z, dz, s
        (+ b, db, ddb, aj, dj if l_mag, xi if l_chem).  ``prof``: or2, or4, orho1, orho2,
        delxr2, delxh2 over the n_r levels.  Returns (outputs dict, dtrkc, dthkc); outputs
        are (lm_max, n_r) with boundary columns zero.  LFfac_r: optional per-level
        Lorentz factor replacing LFfac (levels of several runs in one call).
        """
        w = fields["w"]
        n_r = w.shape[1]
        names = ["w", "dw", "ddw", "z", "dz", "s"] + (["b", "db", "ddb", "aj", "dj"] if l_mag
                                                       else []) + (["xi"] if l_chem else [])
        ins = {}
        for k in names:
            x = fields[k]
            if x.shape != (self.lm_max, n_r) or x.dtype != _CD or x.device != self.device:
                raise ValueError(f"fields[{k}]: expected ({self.lm_max}, {n_r}) complex128")
            ins[k] = x.contiguous()
        onames = ["Advr", "Advt", "Advp", "VSr", "VSt"] + (["VxBr", "VxBt", "VxBp"] if l_mag
                                                           else []) + \
            (["VXir", "VXit"] if l_chem else [])
        if out is None:
            out = {k: torch.zeros(self.lm_max, n_r, dtype=_CD, device=self.device) for k in onames}
        keep = {k: self._prof(prof[k], n_r) for k in
                ("or2", "or4", "orho1", "orho2", "delxr2", "delxh2")}
        bi = _lib.BoussIn(*[ins[k].data_ptr() if k in ins else None for k in
                            ("w", "dw", "ddw", "z", "dz", "s", "b", "db", "ddb", "aj", "dj",
                             "xi")], n_r)
        bo = _lib.BoussOut(*[out[k].data_ptr() if k in out else None for k in
                             ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp",
                              "VXir", "VXit")], out["Advr"].stride(0))
        lf_r = None
        if LFfac_r is not None:
            lf_r = self._prof(LFfac_r, n_r)
            if lf_r.numel() != n_r:
                raise ValueError(f"LFfac_r: expected {n_r} per-level values")
        bp = _lib.BoussParams(*[k.data_ptr() for k in keep.values()], float(LFfac),
                              float(courfac), float(alffac), float(opm), int(l_mag),
                              int(l_chem), (1 if damp else 2) if l_mag else 0, int(parts),
                              lf_r.data_ptr() if lf_r is not None else None)
        dtr = torch.empty(n_r, dtype=_RD, device=self.device)
        dth = torch.empty_like(dtr)
        L = _lib.lib()
        need = L.mt_nl_bouss_workspace(self._h, n_r, int(l_mag), int(l_chem))
        if work is None or work.numel() < need:
            work = self._work(need)
        check(L.mt_nl_bouss(self._h, n_r, C.byref(bi), C.byref(bo), C.byref(bp), _ptr(dtr),
                            _ptr(dth), _ptr(work), work.numel(), self._stream()))
        self._watch(work, "nl_bouss", fused=True)
        return out, dtr, dth

    def get_td(self, ins, prof, CorFac, D1, l_double_curl=False, l_heat=True, l_mag=True,
               l_chem=False, l_anel=False, out=None):
        """Explicit time-derivative terms of one step (magic_torch/step_time.py:1139-1176):
        get_dwdt or get_dwdt_double_curl, get_dzdt, get_dpdt, get_dsdt, get_dxidt and
        get_dbdt (magic_torch/get_td.py:58-308) completed by finish_exp_pol, _entropy,
        _comp and _mag (update_wp.py:371-385, update_s.py:191-210, update_xi.py:183-202,
        update_b.py:514-528), in one launch.

        ``ins``: dict of (lm_max, n_r) complex128 arrays Advr, Advt, Advp, w, dw, z (plus
        ddw, dz for the double-curl form; VSr, VSt if l_heat; VxBr, VxBt, VxBp if l_mag;
        VXir, VXit if l_chem; optionally heat, the anelastic stage's spectral heating,
        added to the entropy term).  ``prof``: r, or1, or2, or4, orho1, beta over n_r.
        ``D1``: the first-derivative RadialOp.  Returns a dict dwdt, dzdt (+ dpdt without
        the double-curl form, dsdt, dxidt, dbdt, djdt as enabled)."""
        n_r = ins["w"].shape[1]
        need = ["Advr", "Advt", "Advp", "w", "dw", "z"]
        need += ["ddw", "dz"] if l_double_curl else []
        need += ["VSr", "VSt"] if l_heat else []
        need += ["VxBr", "VxBt", "VxBp"] if l_mag else []
        need += ["VXir", "VXit"] if l_chem else []
        need += ["heat"] if l_heat and ins.get("heat") is not None else []
        src = {}
        for k in need:
            x = ins[k]
            if x.shape != (self.lm_max, n_r) or x.dtype != _CD or x.device != self.device:
                raise ValueError(f"ins[{k}]: expected ({self.lm_max}, {n_r}) complex128")
            src[k] = x.contiguous()
        onames = ["dwdt", "dzdt"] + ([] if l_double_curl else ["dpdt"]) + \
            (["dsdt"] if l_heat else []) + (["dxidt"] if l_chem else []) + \
            (["dbdt", "djdt"] if l_mag else [])
        if out is None:
            out = {k: torch.empty(self.lm_max, n_r, dtype=_CD, device=self.device)
                   for k in onames}
        keep = {k: self._prof(prof[k], n_r) for k in ("r", "or1", "or2", "or4", "orho1", "beta")}
        ti = _lib.TdIn(*[src[k].data_ptr() if k in src else None for k in
                         ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp", "VXir",
                          "VXit", "w", "dw", "ddw", "z", "dz")], n_r,
                        src["heat"].data_ptr() if "heat" in src else None)
        to = _lib.TdOut(*[out[k].data_ptr() if k in out else None for k in
                          ("dwdt", "dzdt", "dpdt", "dsdt", "dxidt", "dbdt", "djdt")],
                        out["dwdt"].stride(0))
        tp = _lib.TdParams(*[keep[k].data_ptr() for k in ("r", "or1", "or2", "or4", "orho1",
                                                          "beta")],
                           float(CorFac), int(l_double_curl), int(l_heat), int(l_mag),
                           int(l_chem), int(l_anel))
        check(_lib.lib().mt_get_td(self._h, n_r, C.byref(ti), C.byref(to), C.byref(tp),
                                   D1._h if D1 is not None else None, self._stream()))
        return out

    def _nl_anel_composed(self, fields, prof, LFfac, ViscHeatFac, OhmLossFac, courfac, alffac,
                          opm, l_mag, l_chem, damp, out):
        """FP64 plans: the anelastic nonlinear stage composed, as the reference's
        radial_loop_anel composes it (step_time.py:1233-1474), from the FP64 transform
        kernels, mt_get_nl_anel and mt_courant, with the grids in device memory:
        s, xi and the magnetic field on every level; velocity, its radial, theta and
        phi derivatives and cvr on the bulk levels (zero on both boundaries); forward
        transforms of the bulk levels; Courant steps from the zero-boundary velocity."""
        n_r = fields["w"].shape[1]
        for k in ["w", "dw", "ddw", "z", "dz", "s"] + (["b", "db", "ddb", "aj", "dj"] if l_mag
                                                       else []) + (["xi"] if l_chem else []):
            x = fields[k]
            if x.shape != (self.lm_max, n_r) or x.dtype != _CD or x.device != self.device:
                raise ValueError(f"fields[{k}]: expected ({self.lm_max}, {n_r}) complex128")
        if n_r < 3:
            raise MagicError("nl_anel needs n_r >= 3")
        shape = (n_r, self.n_theta_max, self.n_phi_max)
        zeros = lambda: torch.zeros(shape, dtype=_RD, device=self.device)
        d = self.dLh.unsqueeze(1)
        o2 = self._prof(prof["or2"], n_r).unsqueeze(0)
        sc = self.scal_to_spat(fields["s"])
        xic = self.scal_to_spat(fields["xi"]) if l_chem else zeros()
        if l_mag:
            br, bt, bp = self.torpol_to_spat(d * fields["b"], fields["db"], fields["aj"])
            cbr, cbt, cbp = self.torpol_to_spat(d * fields["aj"], fields["dj"],
                                                o2 * d * fields["b"] - fields["ddb"])
        else:
            br, bt, bp, cbr, cbt, cbp = (zeros() for _ in range(6))
        bk = slice(1, n_r - 1)
        wb, dwb, ddwb, zb, dzb = (fields[k][:, bk] for k in ("w", "dw", "ddw", "z", "dz"))

        def bulk(*grids):
            res = []
            for x in grids:
                a = zeros()
                a[bk] = x
                res.append(a)
            return res

        vr, vt, vp = bulk(*self.torpol_to_spat(d * wb, dwb, zb))
        dvrdr, dvtdr, dvpdr = bulk(*self.torpol_to_spat(d * dwb, ddwb, dzb))
        (cvr,) = bulk(self.scal_to_spat(d * zb))
        dvrdt, dvrdp = bulk(*self.pol_to_grad_spat(wb))
        ph = self.dPhi.unsqueeze(1)
        _, gt, gp = self.torpol_to_spat(torch.zeros_like(dwb), ph * dwb, ph * zb)
        ost = self.O_sin_theta_E2_grid.unsqueeze(1)
        dvtdp, dvpdp = bulk(gt * ost, gp * ost)
        nl = self.get_nl_anel([vr, vt, vp, dvrdr, dvtdr, dvpdr, dvrdt, dvrdp, dvtdp, dvpdp, cvr,
                               sc, xic, br, bt, bp, cbr, cbt, cbp], prof, LFfac, ViscHeatFac,
                              OhmLossFac, l_mag)
        Advr, Advt, Advp, VSr, VSt, VSp, VxBr, VxBt, VxBp, VXir, VXit, VXip, heat = nl
        onames = ["Advr", "Advt", "Advp", "VSr", "VSt"] + (["VxBr", "VxBt", "VxBp"] if l_mag
                                                           else []) + \
            (["VXir", "VXit"] if l_chem else []) + ["heat"]
        if out is None:
            out = {k: torch.zeros(self.lm_max, n_r, dtype=_CD, device=self.device) for k in onames}

        def put(name, x):
            out[name][:, 0] = 0.0
            out[name][:, -1] = 0.0
            out[name][:, bk] = x

        put("Advr", self.scal_to_SH(Advr[bk]))
        put("VSr", self.scal_to_SH(VSr[bk]))
        S, T = self.spat_to_sphertor(Advt[bk], Advp[bk])
        put("Advt", S)
        put("Advp", T)
        put("VSt", self.spat_to_sphertor(VSt[bk], VSp[bk])[0])
        if l_mag:
            put("VxBr", self.scal_to_SH(VxBr[bk]))
            S, T = self.spat_to_sphertor(VxBt[bk], VxBp[bk])
            put("VxBt", S)
            put("VxBp", T)
        if l_chem:
            put("VXir", self.scal_to_SH(VXir[bk]))
            put("VXit", self.spat_to_sphertor(VXit[bk], VXip[bk])[0])
        put("heat", self.scal_to_SH(heat[bk]))
        dtr, dth = self.courant(vr, vt, vp, br if l_mag else None, bt, bp, prof, courfac, alffac,
                                LFfac, opm, damp=damp)
        return out, dtr, dth

    def nl_anel_workspace(self, n_r, l_mag=True, l_chem=False):
        return _lib.lib().mt_nl_anel_workspace(self._h, int(n_r), int(l_mag), int(l_chem))

    def nl_anel(self, fields, prof, LFfac, ViscHeatFac, OhmLossFac, courfac, alffac, opm,
                l_mag=True, l_chem=False, damp=True, out=None, work=None):
        """Anelastic nonlinear stage (magic_torch/step_time.py:1215-1475: transforms,
        get_nl_anel with viscous and Ohmic heating, forward transforms, CFL): fused into
        the tcgen05 pack/GEMM and FP32 phi kernels on split-precision plans, into the
        int8 digit-plane GEMMs and an FP64 phi kernel on digit-split (ozaki) plans, and
        composed from the FP64 kernels on FP64 plans (and on a digit-split plan whose
        phi rows would not fit one CTA's shared memory, which no plan within the
        library's n_phi limit reaches).

        ``fields``: dict of spectral (lm_max, n_r) complex128 arrays w, dw, ddw, z, dz, s
        (+ b, db, ddb, aj, dj if l_mag, xi if l_chem).  ``prof``: r, or1, or2, or4, beta,
        orho1, orho2, otemp1, visc, lambda_, delxr2, delxh2 over the n_r levels.  Returns
        (outputs dict Advr Advt Advp VSr VSt [VxBr VxBt VxBp] [VXir VXit] heat, dtrkc,
        dthkc); outputs are (lm_max, n_r) with boundary columns zero.
        """
        w = fields["w"]
        n_r = w.shape[1]
        L = _lib.lib()
        need = L.mt_nl_anel_workspace(self._h, n_r, int(l_mag), int(l_chem)) if n_r >= 3 else 0
        if self.precision == "fp64" or (self.precision == "ozaki" and need == 0):
            return self._nl_anel_composed(fields, prof, LFfac, ViscHeatFac, OhmLossFac, courfac,
                                          alffac, opm, l_mag, l_chem, damp, out)
        if need == 0:
            raise MagicError("nl_anel needs n_r >= 3")
        names = ["w", "dw", "ddw", "z", "dz", "s"] + (["b", "db", "ddb", "aj", "dj"] if l_mag
                                                       else []) + (["xi"] if l_chem else [])
        ins = {}
        for k in names:
            x = fields[k]
            if x.shape != (self.lm_max, n_r) or x.dtype != _CD or x.device != self.device:
                raise ValueError(f"fields[{k}]: expected ({self.lm_max}, {n_r}) complex128")
            ins[k] = x.contiguous()
        onames = ["Advr", "Advt", "Advp", "VSr", "VSt"] + (["VxBr", "VxBt", "VxBp"] if l_mag
                                                           else []) + \
            (["VXir", "VXit"] if l_chem else []) + ["heat"]
        if out is None:
            out = {k: torch.zeros(self.lm_max, n_r, dtype=_CD, device=self.device) for k in onames}
        pnames = ("r", "or1", "or2", "or4", "beta", "orho1", "orho2", "otemp1", "visc",
                  "lambda_", "delxr2", "delxh2")
        keep = {k: self._prof(prof[k], n_r) for k in pnames}
        ai = _lib.AnelIn(*[ins[k].data_ptr() if k in ins else None for k in
                           ("w", "dw", "ddw", "z", "dz", "s", "xi", "b", "db", "ddb", "aj",
                            "dj")], n_r)
        ao = _lib.AnelOut(*[out[k].data_ptr() if k in out else None for k in
                            ("Advr", "Advt", "Advp", "VSr", "VSt", "VxBr", "VxBt", "VxBp",
                             "VXir", "VXit", "heat")], out["Advr"].stride(0))
        ap = _lib.AnelStageParams(*[keep[k].data_ptr() for k in pnames], float(LFfac),
                                  float(ViscHeatFac), float(OhmLossFac), float(courfac),
                                  float(alffac), float(opm), int(l_mag), int(l_chem),
                                  (1 if damp else 2) if l_mag else 0)
        dtr = torch.empty(n_r, dtype=_RD, device=self.device)
        dth = torch.empty_like(dtr)
        if work is None or work.numel() < need:
            work = self._work(need)
        check(L.mt_nl_anel(self._h, n_r, C.byref(ai), C.byref(ao), C.byref(ap), _ptr(dtr),
                           _ptr(dth), _ptr(work), work.numel(), self._stream()))
        self._watch(work, "nl_anel", fused=True)
        return out, dtr, dth
