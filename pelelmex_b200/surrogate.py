"""Learned surrogate of the HP reaction advance and the hybrid reactor.

The surrogate is an MLP that predicts the state change over dt_react:

    x = (T, log10(Y_k + 1e-20) for k < N, log10 dt)          N + 2 inputs
    x -> 256 -> 256 -> 256 (GELU) -> (dT, dY_k)              N + 1 outputs

inputs and outputs standardised by training-set statistics, BF16 weights and
activations with FP32 accumulation.  Every matrix product of inference and
training runs on the tensor cores through the library's hand-written tcgen05
GEMM (b200chem_mlp_gemm_bf16) with fused bias / GELU / GELU-backward
epilogues; the network input and the acceptance gate are library kernels too
(b200chem_surrogate_features, b200chem_surrogate_gate).  PyTorch holds the
device buffers and does the transposes, reductions and the Adam update.

It is trained on (state, dt) -> state pairs labelled by the plain GPU BDF of
the same reactor.  The hybrid reactor predicts every cell, accepts a
prediction only when the gate's conservation, energy and one-step residual
checks pass, and integrates the rejected cells with the BDF.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import mechanism as mechmod

HIDDEN = 256
EPI_F32, EPI_BF16, EPI_GELU, EPI_DGELU = 0, 1, 2, 3


def _torch():
    import torch
    return torch


def _pad16(v: int) -> int:
    return (v + 15) // 16 * 16


def _stream():
    return _torch().cuda.current_stream().cuda_stream


class GemmError(RuntimeError):
    pass


def gemm(A, B, C, bias=None, epi=EPI_F32, aux=None, n_valid=0, err=None):
    """C = epi(A . B^T + bias) on the tensor cores (see b200chem_mlp_gemm_bf16)."""
    M, K = A.shape
    N = B.shape[0]
    code = _lib.load().b200chem_mlp_gemm_bf16(
        A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K, C.data_ptr(), C.stride(0),
        bias.data_ptr() if bias is not None else None, aux.data_ptr() if aux is not None else None, epi, n_valid,
        err.data_ptr() if err is not None else None, _stream())
    if code != 0:
        raise GemmError(f"tensor-core GEMM rejected M={M} N={N} K={K} epi={epi} (code {code})")
    return C


@dataclass
class GateOpts:
    """Acceptance thresholds (b200chem_gate_opts).  The defaults keep the
    accepted cells of the drm19-shaped flame field within 1e-4 relative T of
    the BDF with margin (held-out seeded cells, two-member ensemble): raw mass
    and element errors below 1e-3 (then corrected exactly), T from (h, Y)
    within 0.05 K of the predicted T, predicted |dT| <= 0.2 K, and the
    one-step implicit residual of the temperature within 10 % of its change."""
    rtol: float = 1e-6
    atol: float = 0.0
    tol_T: float = 0.05
    tol_elem: float = 1e-3
    tol_mass: float = 1e-3
    rchange: float = 0.1
    dT_max: float = 0.2
    t_source: int = 1
    residual_t_only: int = 1

    def ctypes(self):
        return _lib.GateOpts(self.rtol, self.atol, self.tol_T, self.tol_elem, self.tol_mass, self.rchange,
                             self.dT_max, self.t_source, self.residual_t_only)


class MLPSurrogate:
    """The network, its normalisation, and its tensor-core training."""

    def __init__(self, mech, seed: int = 0, device="cuda:0"):
        torch = _torch()
        if isinstance(mech, str):
            mech = mechmod.builtin(mech)
        self.mech = mech
        self.N = mech.n_species
        self.nin, self.nout = self.N + 2, self.N + 1
        self.kin, self.kout = _pad16(self.nin), _pad16(self.nout)
        self.device = torch.device(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        dims = [(HIDDEN, self.kin, self.nin), (HIDDEN, HIDDEN, HIDDEN), (HIDDEN, HIDDEN, HIDDEN),
                (self.kout, HIDDEN, HIDDEN)]
        self.W, self.b = [], []
        for li, (o, i, fan_in) in enumerate(dims):
            W = torch.zeros((o, i))
            lim = math.sqrt(6.0 / fan_in) if li < 3 else math.sqrt(3.0 / fan_in)
            rows = o if li < 3 else self.nout
            W[:rows, :fan_in] = (torch.rand((rows, fan_in), generator=g) * 2 - 1) * lim
            self.W.append(W.to(self.device))
            self.b.append(torch.zeros(o, device=self.device))
        self.xmean = torch.zeros(self.nin, device=self.device)
        self.xstd = torch.ones(self.nin, device=self.device)
        self.ymean = torch.zeros(self.nout, device=self.device)
        self.ystd = torch.ones(self.nout, device=self.device)
        self._adam = None
        self._sync_bf16()

    # ------------------------------------------------------------ weights
    def _sync_bf16(self):
        torch = _torch()
        self.Wb = [W.to(torch.bfloat16).contiguous() for W in self.W]
        self.WbT = [W.t().contiguous() for W in self.Wb]

    def state_dict(self):
        return {"W": [W.cpu() for W in self.W], "b": [b.cpu() for b in self.b], "xmean": self.xmean.cpu(),
                "xstd": self.xstd.cpu(), "ymean": self.ymean.cpu(), "ystd": self.ystd.cpu(), "N": self.N}

    def load_state_dict(self, d):
        self.W = [W.to(self.device) for W in d["W"]]
        self.b = [b.to(self.device) for b in d["b"]]
        for k in ("xmean", "xstd", "ymean", "ystd"):
            setattr(self, k, d[k].to(self.device))
        self._sync_bf16()

    # ----------------------------------------------------------- features
    def raw_features(self, rhoY, T, dt):
        """Unstandardised inputs [ncells, N + 2] (FP32, for statistics)."""
        torch = _torch()
        Y = rhoY / rhoY.sum(dim=0, keepdim=True)
        lg = torch.log10(Y.clamp_min(0.0) + 1e-20)
        dtc = torch.full_like(T, math.log10(dt))
        return torch.cat([T[None], lg, dtc[None]]).t().float()

    def features(self, reactor, rhoY, T, dt, nrows):
        """Standardised BF16 network input [nrows, kin] (library kernel)."""
        torch = _torch()
        x = torch.empty((nrows, self.kin), dtype=torch.bfloat16, device=self.device)
        _lib.check(_lib.load().b200chem_surrogate_features(
            reactor._h, rhoY.data_ptr(), T.data_ptr(), T.shape[0], nrows, float(dt), self.xmean.data_ptr(),
            self.xstd.data_ptr(), x.data_ptr(), _stream()))
        return x

    # ------------------------------------------------------------ forward
    def forward(self, x, train=False):
        """x: [B, kin] BF16 (B % 128 == 0) -> standardised outputs [B, kout] FP32."""
        torch = _torch()
        B = x.shape[0]
        err = torch.zeros(1, dtype=torch.int32, device=self.device)
        acts, pres = [x], []
        h = x
        for li in range(3):
            pre = torch.empty((B, HIDDEN), dtype=torch.float32, device=self.device) if train else None
            out = torch.empty((B, HIDDEN), dtype=torch.bfloat16, device=self.device)
            gemm(h, self.Wb[li], out, self.b[li], EPI_GELU, aux=pre, err=err)
            acts.append(out)
            pres.append(pre)
            h = out
        y = torch.zeros((B, self.kout), dtype=torch.float32, device=self.device)
        gemm(h, self.Wb[3], y, self.b[3], EPI_F32, n_valid=self.nout, err=err)
        self._err = err
        return (y, (acts, pres)) if train else y

    def check_error(self):
        if int(self._err.item()) != 0:
            raise GemmError("a tensor-core completion wait timed out")

    # ----------------------------------------------------------- backward
    def loss_and_grads(self, x, target, weights):
        """Weighted MSE on standardised outputs; gradients by the tensor cores."""
        torch = _torch()
        B = x.shape[0]
        y, (acts, pres) = self.forward(x, train=True)
        diff = (y[:, :self.nout] - target) * weights
        loss = (diff * (y[:, :self.nout] - target)).sum() / B
        d = torch.zeros((B, self.kout), dtype=torch.float32, device=self.device)
        d[:, :self.nout] = 2.0 * diff / B
        db = [None] * 4
        dW = [None] * 4
        err = self._err
        dz = d.to(torch.bfloat16)
        for li in range(3, -1, -1):
            db[li] = dz.float().sum(dim=0)
            # dW = dz^T a  (M = out features, padded to 128 rows; K = batch)
            out_f = dz.shape[1]
            mpad = (out_f + 127) // 128 * 128
            dzT = torch.zeros((mpad, B), dtype=torch.bfloat16, device=self.device)
            dzT[:out_f] = dz.t()
            aT = acts[li].t().contiguous()
            Cw = torch.empty((mpad, aT.shape[0]), dtype=torch.float32, device=self.device)
            gemm(dzT, aT, Cw, err=err)
            dW[li] = Cw[:out_f]
            if li > 0:
                # dz_prev = (dz W) * gelu'(pre_prev)
                nxt = torch.empty((B, HIDDEN), dtype=torch.bfloat16, device=self.device)
                gemm(dz, self.WbT[li], nxt, None, EPI_DGELU, aux=pres[li - 1], err=err)
                dz = nxt
        return loss, dW, db

    def adam_step(self, dW, db, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        torch = _torch()
        if self._adam is None:
            self._adam = {"t": 0, "m": [torch.zeros_like(p) for p in self.W + self.b],
                          "v": [torch.zeros_like(p) for p in self.W + self.b]}
        st = self._adam
        st["t"] += 1
        c1 = 1 - beta1 ** st["t"]
        c2 = 1 - beta2 ** st["t"]
        params = self.W + self.b
        grads = list(dW) + list(db)
        for p, g, m, v in zip(params, grads, st["m"], st["v"]):
            m.mul_(beta1).add_(g, alpha=1 - beta1)
            v.mul_(beta2).addcmul_(g, g, value=1 - beta2)
            p.addcdiv_(m / c1, (v / c2).sqrt_().add_(eps), value=-lr)
        # keep the padding exactly zero
        self.W[0][:, self.nin:] = 0
        self.W[3][self.nout:] = 0
        self.b[3][self.nout:] = 0
        self._sync_bf16()

    # ----------------------------------------------------------- training
    def fit_normalisation(self, raw_x, dy):
        torch = _torch()
        self.xmean = raw_x.mean(dim=0)
        self.xstd = raw_x.std(dim=0).clamp_min(1e-3)
        self.ymean = dy.mean(dim=0)
        floor = torch.full_like(self.ymean, 1e-12)
        floor[0] = 1e-6
        self.ystd = torch.maximum(dy.std(dim=0), floor)

    def train(self, x_all, y_all, steps=4000, batch=8192, lr=2e-3, lr_end=2e-5, weights=None, log_every=0,
              seed=0):
        """x_all [S, kin] BF16 standardised inputs; y_all [S, nout] FP32 standardised targets."""
        torch = _torch()
        S = x_all.shape[0]
        if weights is None:
            weights = torch.ones(self.nout, device=self.device)
            weights[0] = 4.0
        g = torch.Generator(device=self.device).manual_seed(seed)
        hist = []
        for it in range(steps):
            idx = torch.randint(0, S, (batch,), device=self.device, generator=g)
            lr_t = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * it / max(1, steps - 1)))
            loss, dW, db = self.loss_and_grads(x_all[idx], y_all[idx], weights)
            self.adam_step(dW, db, lr_t)
            if log_every and (it % log_every == 0 or it == steps - 1):
                hist.append((it, float(loss.item())))
        self.check_error()
        return hist

    def standardise_targets(self, dy):
        return (dy - self.ymean) / self.ystd


def element_matrix(mech):
    return np.ascontiguousarray(mech.element_matrix(), dtype=np.float64)


def label_pairs(reactor, field, device="cuda:0"):
    """Inputs and BDF-labelled changes for every cell of a field: returns
    (rhoY0, T0, dy) with dy [ncells, N + 1] = (T1 - T0, Y1 - Y0)."""
    torch = _torch()
    rhoY = torch.tensor(field.rhoY, device=device)
    T = torch.tensor(field.T, device=device)
    rhoH = torch.tensor(field.rhoH, device=device)
    fY = torch.zeros_like(rhoY)
    fH = torch.zeros_like(T)
    rY1, T1, rH1 = rhoY.clone(), T.clone(), rhoH.clone()
    reactor.react_flat(rY1, fY, T1, rH1, fH, dt_react=field.dt)
    Y0 = rhoY / rhoY.sum(dim=0, keepdim=True)
    Y1 = rY1 / rY1.sum(dim=0, keepdim=True)
    dy = torch.cat([(T1 - T)[None], Y1 - Y0]).t().contiguous().float()
    return rhoY, T, dy


class HybridReactor:
    """Surrogate-first reaction advance with gated fallback to the BDF.

    `surrogate` is one network or a list of networks sharing one
    normalisation (an ensemble): with several, the gate sees their mean
    prediction and a cell whose members disagree on dT by more than
    tol_ensemble (K) is rejected before the conservation / energy / residual
    checks."""

    def __init__(self, reactor, surrogate, gate: GateOpts | None = None, tol_ensemble: float = 0.05):
        torch = _torch()
        self.r = reactor
        self.members = list(surrogate) if isinstance(surrogate, (list, tuple)) else [surrogate]
        self.s = self.members[0]
        self.gate = gate or GateOpts()
        self.tol_ensemble = tol_ensemble
        self.elem = torch.tensor(element_matrix(self.s.mech), device=self.s.device)
        self.last = {}

    def react_flat(self, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount=None, dt_react=1e-6):
        torch = _torch()
        nc = T.shape[0]
        if nc == 0:
            return 0
        nrows = (nc + 127) // 128 * 128
        x = self.s.features(self.r, rhoY, T, dt_react, nrows)
        pred = self.s.forward(x)
        if len(self.members) > 1:
            preds = [pred] + [m.forward(x) for m in self.members[1:]]
            pred = torch.stack(preds).mean(dim=0)
            spread = torch.stack([(p[:, 0] - pred[:, 0]).abs() for p in preds]).amax(dim=0) * self.s.ystd[0]
            pred[spread > self.tol_ensemble, 0] = float("nan")  # the gate rejects a non-finite dT
        accept = torch.empty(nc, dtype=torch.int32, device=T.device)
        go = self.gate.ctypes()
        _lib.check(_lib.load().b200chem_surrogate_gate(
            self.r._h, rhoY.data_ptr(), extF_rhoY.data_ptr(), T.data_ptr(), rhoH.data_ptr(), extF_rhoH.data_ptr(),
            fctCount.data_ptr() if fctCount is not None else None, nc, float(dt_react), pred.data_ptr(),
            self.s.ymean.data_ptr(), self.s.ystd.data_ptr(), self.elem.data_ptr(), self.elem.shape[0],
            ctypes.byref(go), accept.data_ptr(), _stream()))
        rej = torch.nonzero(accept != 1).flatten()
        nrej = int(rej.numel())
        if nrej:
            rY = rhoY.index_select(1, rej).contiguous()
            fY = extF_rhoY.index_select(1, rej).contiguous()
            Tr = T.index_select(0, rej).contiguous()
            rH = rhoH.index_select(0, rej).contiguous()
            fH = extF_rhoH.index_select(0, rej).contiguous()
            fc = torch.zeros(nrej, dtype=torch.float64, device=T.device)
            self.r.react_flat(rY, fY, Tr, rH, fH, fc, dt_react=dt_react)
            rhoY.index_copy_(1, rej, rY)
            T.index_copy_(0, rej, Tr)
            rhoH.index_copy_(0, rej, rH)
            if fctCount is not None:
                fctCount.index_copy_(0, rej, fc + 2.0)
        counts = torch.bincount((-accept).clamp_min(0), minlength=6).tolist()
        self.last = {"cells": nc, "rejected": nrej, "accepted_fraction": 1.0 - nrej / nc, "accepted": accept == 1,
                     "rejected_by": {"mass": counts[1], "elements": counts[2], "energy": counts[3],
                                     "residual": counts[4], "change": counts[5]}}
        return nrej


def train_ensemble(reactor, mech, fields, members=2, steps=4000, batch=8192, lr=2e-3, seed=0):
    """Label every cell of `fields` with the BDF, fit one normalisation and
    train `members` networks (different initialisations and batch orders)."""
    torch = _torch()
    rhoYs, Ts, dys, dts = [], [], [], []
    for f in fields:
        rY, T, dy = label_pairs(reactor, f)
        rhoYs.append(rY)
        Ts.append(T)
        dys.append(dy)
        dts.append(f.dt)
    nets = []
    s0 = MLPSurrogate(mech, seed=seed)
    raw = torch.cat([s0.raw_features(rY, T, dt) for rY, T, dt in zip(rhoYs, Ts, dts)])
    dy = torch.cat(dys)
    s0.fit_normalisation(raw, dy)
    xs = []
    for rY, T, dt in zip(rhoYs, Ts, dts):
        nc = T.shape[0]
        xs.append(s0.features(reactor, rY, T, dt, (nc + 127) // 128 * 128)[:nc])
    x = torch.cat(xs)
    y = s0.standardise_targets(dy)
    for mbr in range(members):
        s = s0 if mbr == 0 else MLPSurrogate(mech, seed=seed + mbr)
        if mbr:
            s.xmean, s.xstd, s.ymean, s.ystd = s0.xmean, s0.xstd, s0.ymean, s0.ystd
        s.train(x, y, steps=steps, batch=batch, lr=lr, seed=seed + 7 * mbr)
        nets.append(s)
    return nets
