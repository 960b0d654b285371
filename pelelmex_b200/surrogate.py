"""Learned surrogate of the HP reaction advance and the hybrid reactor.

The surrogate is an ensemble of MLPs that predict the state change over
dt_react:

    x = (T, log10(Y_k + 1e-20) for k < N, log10 dt)          N + 2 inputs
    x -> 256 -> 256 -> 256 (GELU) -> (dT, dY_k)              N + 1 outputs

Inputs are standardised by training-set statistics.  Outputs are
u_j = asinh(dy_j / s_j) (s_T = 0.02 K, s_k a tenth of the median |dY_k| of the
training pairs), standardised: the transform gives every decade of change the
same resolution, so a 0.5 K and a 50 K temperature change are learnt to the
same relative accuracy.

Precision: BF16 weights, FP32 accumulation on the tensor cores (the
library's hand-written tcgen05 GEMM, b200chem_mlp_gemm_bf16).  Inputs and
hidden activations travel as two BF16 terms (hi = bf16(v), lo = bf16(v - hi),
about 16 significant bits): a single BF16 term resolves T only to ~2 K and
log10 Y to ~0.01, which alone moves the predicted dT of flame cells by several
times the 1e-4 relative bar.  Both terms are multiplied by the same weights
and summed in the FP32 accumulator.

Training runs on the GPU through the same GEMMs (forward, dz = (dz W) *
gelu'(pre), dW = dz^T a) and a fused Adam kernel (b200chem_mlp_adam); PyTorch
holds the buffers and does the transposes and bias-gradient sums.  Training
pairs are (state, dt) -> state labelled by the plain GPU BDF of the same
reactor.

The hybrid reactor (b200chem_react_hybrid) predicts every cell with every
member, accepts a prediction only when the ensemble agrees within a fraction
of the temperature bar, the change is within the range where the ensemble's
agreement bounds its error, the raw prediction conserves mass and elements,
T from (h, Y) agrees with the predicted T, and a one-step implicit residual
holds; accepted cells get the element- and energy-consistent state, the
others are integrated by the BDF, all in one library call.
"""
from __future__ import annotations

import ctypes
import math
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from . import mechanism as mechmod

HIDDEN = 256
EPI_F32, EPI_BF16, EPI_GELU, EPI_DGELU = 0, 1, 2, 3
SPLIT_OUT, SPLIT_A = 0x10, 0x20
T_SCALE = 0.02  # K: asinh scale of the temperature change
Y_SCALE_FLOOR = 1e-9  # smallest asinh scale of a mass-fraction change

MAGIC = b"B2CHSURR"
FILE_VERSION = 1
HEADER_BYTES = 256


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
    """C = epi(A . B^T + bias) on the tensor cores (b200chem_mlp_gemm_bf16);
    K is B's row length (A holds two terms of it when SPLIT_A is set)."""
    M = A.shape[0]
    N, K = B.shape
    code = _lib.load().b200chem_mlp_gemm_bf16(
        A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K, C.data_ptr(), C.stride(0),
        bias.data_ptr() if bias is not None else None, aux.data_ptr() if aux is not None else None, epi, n_valid,
        err.data_ptr() if err is not None else None, _stream())
    if code != 0:
        raise GemmError(f"tensor-core GEMM rejected M={M} N={N} K={K} epi={epi:#x} (code {code})")
    return C


@dataclass
class HybridOpts:
    """Acceptance rule of the hybrid reactor (b200chem_hybrid_opts).  All
    temperature bounds are in units of t_rel * T (the error bar itself)."""
    t_rel: float = 1e-4     # relative T error the accepted cells are held to
    spread: float = 0.05    # max deviation of a member's dT from the ensemble mean
    dT_cap: float = 10.0    # max |predicted dT| (the ensemble's shared bias grows with the change)
    gap: float = 5.0        # max |T(h, Y_pred) - T_pred| before the energy projection
    tol_elem: float = 2e-3  # raw element-conservation error, relative to the atom content
    tol_mass: float = 2e-3  # raw mass-conservation error, relative
    resid: float = 0.0      # one-step residual bound (0: off)
    min_members: int = 2

    def ctypes(self):
        return _lib.HybridOpts(self.t_rel, self.spread, self.dT_cap, self.gap, self.tol_elem, self.tol_mass,
                               self.resid, self.min_members, 0)

    def as_tuple(self):
        return (self.t_rel, self.spread, self.dT_cap, self.gap, self.tol_elem, self.tol_mass, self.resid)


class MLPSurrogate:
    """One network of the ensemble and its tensor-core training."""

    def __init__(self, mech, seed: int = 0, device="cuda:0", terms: int = 2):
        torch = _torch()
        if isinstance(mech, str):
            mech = mechmod.builtin(mech)
        self.mech = mech
        self.N = mech.n_species
        self.nin, self.nout = self.N + 2, self.N + 1
        self.kin, self.kout = _pad16(self.nin), _pad16(self.nout)
        self.terms = terms
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
        self.tscale = torch.ones(self.nout, dtype=torch.float64, device=self.device)
        self._adam = None
        self._err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._sync_bf16()

    # ------------------------------------------------------------ weights
    def _sync_bf16(self):
        torch = _torch()
        self.Wb = [W.to(torch.bfloat16).contiguous() for W in self.W]
        self.WbT = [W.t().contiguous() for W in self.Wb]

    def share_normalisation(self, other: "MLPSurrogate"):
        self.xmean, self.xstd, self.ymean, self.ystd, self.tscale = (other.xmean, other.xstd, other.ymean,
                                                                     other.ystd, other.tscale)

    def state_dict(self):
        return {"W": [W.cpu() for W in self.W], "b": [b.cpu() for b in self.b], "xmean": self.xmean.cpu(),
                "xstd": self.xstd.cpu(), "ymean": self.ymean.cpu(), "ystd": self.ystd.cpu(),
                "tscale": self.tscale.cpu(), "N": self.N, "terms": self.terms}

    def load_state_dict(self, d):
        self.W = [W.to(self.device).float() for W in d["W"]]
        self.b = [b.to(self.device).float() for b in d["b"]]
        for k in ("xmean", "xstd", "ymean", "ystd"):
            setattr(self, k, d[k].to(self.device).float())
        self.tscale = d["tscale"].to(self.device).double()
        self.terms = int(d.get("terms", self.terms))
        self._adam = None
        self._sync_bf16()

    # ----------------------------------------------------------- features
    def raw_features(self, rhoY, T, dt):
        """Unstandardised inputs [ncells, N + 2] (FP64, for statistics)."""
        torch = _torch()
        Y = rhoY / rhoY.sum(dim=0, keepdim=True)
        lg = torch.log10(Y.clamp_min(0.0) + 1e-20)
        dtc = torch.full_like(T, math.log10(dt))
        return torch.cat([T[None], lg, dtc[None]]).t()

    def features(self, reactor, rhoY, T, dt, nrows):
        """Standardised BF16 network input [nrows, terms * kin] (library kernel)."""
        torch = _torch()
        x = torch.empty((nrows, self.terms * self.kin), dtype=torch.bfloat16, device=self.device)
        _lib.check(_lib.load().b200chem_surrogate_features(
            reactor._h, rhoY.data_ptr(), T.data_ptr(), T.shape[0], nrows, float(dt), self.xmean.data_ptr(),
            self.xstd.data_ptr(), self.terms, x.data_ptr(), _stream()))
        return x

    # ------------------------------------------------------------ forward
    def forward(self, x, train=False):
        """x: [B, terms * kin] BF16 (B % 128 == 0) -> standardised outputs [B, kout] FP32."""
        torch = _torch()
        B = x.shape[0]
        split = SPLIT_A if self.terms == 2 else 0
        out_split = SPLIT_OUT if self.terms == 2 else 0
        acts, pres = [x], []
        h = x
        for li in range(3):
            pre = torch.empty((B, HIDDEN), dtype=torch.float32, device=self.device) if train else None
            out = torch.empty((B, self.terms * HIDDEN), dtype=torch.bfloat16, device=self.device)
            gemm(h, self.Wb[li], out, self.b[li], EPI_GELU | split | out_split, aux=pre, err=self._err)
            acts.append(out)
            pres.append(pre)
            h = out
        y = torch.zeros((B, self.kout), dtype=torch.float32, device=self.device)
        gemm(h, self.Wb[3], y, self.b[3], EPI_F32 | split, n_valid=self.nout, err=self._err)
        return (y, (acts, pres)) if train else y

    def check_error(self):
        if int(self._err.item()) != 0:
            raise GemmError("a tensor-core completion wait timed out")

    def decode(self, y):
        """Standardised outputs -> physical changes (dT, dY_k) [B, N + 1], FP64."""
        torch = _torch()
        u = y[:, :self.nout].double() * self.ystd.double() + self.ymean.double()
        return torch.sinh(u) * self.tscale

    def encode(self, dy):
        """Physical changes [B, N + 1] -> standardised targets (FP32)."""
        torch = _torch()
        u = torch.asinh(dy / self.tscale)
        return ((u - self.ymean.double()) / self.ystd.double()).float()

    # ----------------------------------------------------------- backward
    def loss_and_grads(self, x, target, weights):
        """Weighted MSE on standardised outputs; gradients by the tensor cores.
        The weight gradients use the high term of each two-term activation."""
        torch = _torch()
        B = x.shape[0]
        y, (acts, pres) = self.forward(x, train=True)
        diff = (y[:, :self.nout] - target) * weights
        loss = (diff * (y[:, :self.nout] - target)).sum() / B
        d = torch.zeros((B, self.kout), dtype=torch.float32, device=self.device)
        d[:, :self.nout] = 2.0 * diff / B
        db = [None] * 4
        dW = [None] * 4
        dz = d.to(torch.bfloat16)
        for li in range(3, -1, -1):
            db[li] = dz.float().sum(dim=0)
            # dW = dz^T a  (M = out features, padded to 128 rows; K = batch)
            out_f = dz.shape[1]
            mpad = (out_f + 127) // 128 * 128
            dzT = torch.zeros((mpad, B), dtype=torch.bfloat16, device=self.device)
            dzT[:out_f] = dz.t()
            width = self.W[li].shape[1]
            aT = acts[li][:, :width].t().contiguous()
            Cw = torch.empty((mpad, width), dtype=torch.float32, device=self.device)
            gemm(dzT, aT, Cw, err=self._err)
            dW[li] = Cw[:out_f].contiguous()
            if li > 0:
                # dz_prev = (dz W) * gelu'(pre_prev)
                nxt = torch.empty((B, HIDDEN), dtype=torch.bfloat16, device=self.device)
                gemm(dz, self.WbT[li], nxt, None, EPI_DGELU, aux=pres[li - 1], err=self._err)
                dz = nxt
        return loss, dW, db

    def adam_step(self, dW, db, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        """One fused Adam step (b200chem_mlp_adam) per tensor; refreshes the BF16 copies."""
        torch = _torch()
        if self._adam is None:
            self._adam = {"t": 0, "m": [torch.zeros_like(p) for p in self.W + self.b],
                          "v": [torch.zeros_like(p) for p in self.W + self.b]}
        st = self._adam
        st["t"] += 1
        L = _lib.load()
        for i, (p, g) in enumerate(zip(self.W + self.b, list(dW) + list(db))):
            rows, cols = (p.shape[0], p.shape[1]) if p.dim() == 2 else (1, p.shape[0])
            wb = self.Wb[i].data_ptr() if i < 4 else None
            wbt = self.WbT[i].data_ptr() if i < 4 else None
            code = L.b200chem_mlp_adam(p.data_ptr(), g.contiguous().data_ptr(), st["m"][i].data_ptr(),
                                       st["v"][i].data_ptr(), rows, cols, float(lr), beta1, beta2, eps, st["t"],
                                       wb, wbt, _stream())
            if code != 0:
                raise GemmError(f"adam step rejected (code {code})")

    # ----------------------------------------------------------- training
    def train(self, x_all, y_all, steps=4000, batch=8192, lr=2e-3, lr_end=2e-5, weights=None, log_every=0,
              seed=0):
        """x_all [S, terms * kin] BF16 standardised inputs; y_all [S, nout] FP32 standardised targets."""
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


def element_matrix(mech):
    return np.ascontiguousarray(mech.element_matrix(), dtype=np.float64)


def label_pairs(reactor, field, device="cuda:0"):
    """Inputs and BDF-labelled changes for every cell of a field: returns
    (rhoY0, T0, dy, fct) with dy [ncells, N + 1] = (T1 - T0, Y1 - Y0) in FP64
    and fct the BDF's right-hand-side count per cell."""
    torch = _torch()
    rhoY = torch.as_tensor(field.rhoY, device=device)
    T = torch.as_tensor(field.T, device=device)
    rhoH = torch.as_tensor(field.rhoH, device=device)
    fY = torch.zeros_like(rhoY)
    fH = torch.zeros_like(T)
    rY1, T1, rH1 = rhoY.clone(), T.clone(), rhoH.clone()
    fct = torch.zeros_like(T)
    reactor.react_flat(rY1, fY, T1, rH1, fH, fct, dt_react=field.dt)
    Y0 = rhoY / rhoY.sum(dim=0, keepdim=True)
    Y1 = rY1 / rY1.sum(dim=0, keepdim=True)
    dy = torch.cat([(T1 - T)[None], Y1 - Y0]).t().contiguous()
    return rhoY, T, dy, fct


class Ensemble:
    """Networks sharing one normalisation, with the acceptance rule they were
    calibrated for; saved in the library's versioned weights format."""

    def __init__(self, members, opts: HybridOpts | None = None):
        self.members = list(members)
        self.s = self.members[0]
        self.opts = opts or HybridOpts()

    @property
    def mech(self):
        return self.s.mech

    def predict(self, reactor, rhoY, T, dt):
        """Decoded predictions of every member, [M, ncells, N + 1] FP64."""
        torch = _torch()
        nc = T.shape[0]
        nrows = (nc + 127) // 128 * 128
        x = self.s.features(reactor, rhoY, T, dt, nrows)
        return torch.stack([m.decode(m.forward(x)[:nc]) for m in self.members])

    # --------------------------------------------------------- file format
    def to_bytes(self) -> bytes:
        """The versioned weights file (layout documented in include/b200chem.h,
        b200chem_surrogate_load)."""
        s = self.s
        flat = mechmod.flatten(s.mech)
        from . import mechgen
        digest = mechgen.mechanism_digest(flat)
        o = self.opts
        hdr = MAGIC + struct.pack("<II", FILE_VERSION, HEADER_BYTES) + struct.pack("<Q", digest)
        elem = element_matrix(s.mech)
        hdr += struct.pack("<12i", s.N, s.nin, s.nout, HIDDEN, s.kin, s.kout, len(self.members), s.terms, 1,
                           int(o.min_members), elem.shape[0], 0)
        hdr += struct.pack("<7d", *o.as_tuple())
        hdr += b"\0" * (HEADER_BYTES - len(hdr))
        assert len(hdr) == HEADER_BYTES
        body = b"".join(np.ascontiguousarray(t.detach().cpu().numpy(), dtype=np.float32).tobytes()
                        for t in (s.xmean, s.xstd, s.ymean, s.ystd))
        body += np.ascontiguousarray(s.tscale.cpu().numpy(), dtype=np.float64).tobytes()
        body += elem.tobytes()
        for m in self.members:
            for li in range(4):
                body += m.Wb[li].contiguous().cpu().view(_torch().int16).numpy().tobytes()
                body += np.ascontiguousarray(m.b[li].cpu().numpy(), dtype=np.float32).tobytes()
        return hdr + body

    def save(self, path):
        Path(path).write_bytes(self.to_bytes())

    @classmethod
    def from_bytes(cls, data: bytes, mech, device="cuda:0") -> "Ensemble":
        torch = _torch()
        if data[:8] != MAGIC:
            raise ValueError("not a surrogate weights file (bad magic)")
        version, hbytes = struct.unpack_from("<II", data, 8)
        if version != FILE_VERSION:
            raise ValueError(f"surrogate weights file version {version}, expected {FILE_VERSION}")
        (digest,) = struct.unpack_from("<Q", data, 16)
        N, nin, nout, hidden, kin, kout, M, terms, dtype, min_members, ne, _ = struct.unpack_from("<12i", data, 24)
        opts = struct.unpack_from("<7d", data, 72)
        if isinstance(mech, str):
            mech = mechmod.builtin(mech)
        from . import mechgen
        if mechgen.mechanism_digest(mechmod.flatten(mech)) != digest:
            raise ValueError("surrogate weights were trained for a different mechanism (digest mismatch)")
        if hidden != HIDDEN or N != mech.n_species or dtype != 1:
            raise ValueError("surrogate weights file has unsupported dimensions or dtype")
        off = hbytes

        def take(n, dt):
            nonlocal off
            a = np.frombuffer(data, dtype=dt, count=n, offset=off).copy()
            off += n * np.dtype(dt).itemsize
            return a
        norm = [torch.tensor(take(n, np.float32), device=device) for n in (nin, nin, nout, nout)]
        tscale = torch.tensor(take(nout, np.float64), device=device)
        take(ne * N, np.float64)  # element matrix: the library's gate reads it; here it follows from mech
        members = []
        dims = [(hidden, kin), (hidden, hidden), (hidden, hidden), (kout, hidden)]
        for _ in range(M):
            m = MLPSurrogate(mech, device=device, terms=terms)
            for li, (r, c) in enumerate(dims):
                w = torch.from_numpy(take(r * c, np.int16).reshape(r, c)).view(torch.bfloat16)
                m.W[li] = w.float().to(device)
                m.b[li] = torch.tensor(take(r, np.float32), device=device)
            m.xmean, m.xstd, m.ymean, m.ystd = norm
            m.tscale = tscale
            m._sync_bf16()
            members.append(m)
        if off != len(data):
            raise ValueError("surrogate weights file has trailing or missing bytes")
        return cls(members, HybridOpts(*opts, min_members=min_members))

    @classmethod
    def load(cls, path, mech, device="cuda:0") -> "Ensemble":
        return cls.from_bytes(Path(path).read_bytes(), mech, device)


def fit_normalisation(s: MLPSurrogate, raw_x, dy):
    """Input statistics, asinh scales and output statistics from training pairs."""
    torch = _torch()
    s.xmean = raw_x.mean(dim=0).float()
    s.xstd = raw_x.std(dim=0).clamp_min(1e-3).float()
    n = dy.shape[0]
    sub = dy[torch.randperm(n, device=dy.device)[:min(n, 500_000)]]
    # species: a tenth of the median change, floored at 1e-9 -- changes of Y
    # below that are at the BDF's own absolute tolerance (atol 1e-12 on
    # rho Y, rho ~ 1e-3 g/cm^3) and carry no temperature information
    sY = (sub[:, 1:].abs().median(dim=0).values * 0.1).clamp_min(Y_SCALE_FLOOR)
    s.tscale = torch.cat([torch.tensor([T_SCALE], dtype=torch.float64, device=dy.device), sY])
    u = torch.asinh(dy / s.tscale)
    s.ymean = u.mean(dim=0).float()
    s.ystd = u.std(dim=0).float().clamp_min(1e-6)


def train_ensemble(reactor, mech, fields, members=4, steps=8000, batch=16384, lr=2e-3, seed=0, t_weight=None,
                   bag=0.8, terms=2, log=None):
    """Label every cell of `fields` with the BDF, fit one normalisation and
    train `members` networks, each on its own random share `bag` of the pairs
    (different initialisations and batch orders)."""
    torch = _torch()
    raws, dys, xs_src = [], [], []
    s0 = MLPSurrogate(mech, seed=seed, terms=terms)
    for f in fields:
        rY, T, dy, _ = label_pairs(reactor, f)
        raws.append(s0.raw_features(rY, T, f.dt))
        dys.append(dy)
        xs_src.append((rY, T, f.dt))
    dy = torch.cat(dys)
    fit_normalisation(s0, torch.cat(raws), dy)
    del raws
    xs = []
    for rY, T, dt in xs_src:
        nc = T.shape[0]
        xs.append(s0.features(reactor, rY, T, dt, (nc + 127) // 128 * 128)[:nc])
    del xs_src
    x = torch.cat(xs)
    y = s0.encode(dy)
    del xs, dy
    w = torch.ones(s0.nout, device=s0.device)
    w[0] = float(t_weight if t_weight is not None else s0.N)
    S = x.shape[0]
    nets = []
    for mbr in range(members):
        s = s0 if mbr == 0 else MLPSurrogate(mech, seed=seed + mbr, terms=terms)
        s.share_normalisation(s0)
        if bag < 1.0:
            gen = torch.Generator(device=s.device).manual_seed(1000 + seed + mbr)
            sub = torch.randperm(S, device=s.device, generator=gen)[: int(bag * S)]
            xm, ym = x[sub], y[sub]
        else:
            xm, ym = x, y
        hist = s.train(xm, ym, steps=steps, batch=batch, lr=lr, weights=w, seed=seed + 7 * mbr,
                       log_every=max(1, steps // 4))
        if log:
            log(f"member {mbr}: loss {[round(h[1], 5) for h in hist]}")
        nets.append(s)
        del xm, ym
    return nets


def finetune_ensemble(reactor, ens, fields, steps=8000, batch=16384, lr=2e-4, lr_end=2e-6, seed=100, t_weight=None,
                      bag=0.8, log=None):
    """Continue training every member of `ens` on BDF-labelled `fields`, in
    the ensemble's own normalisation (inputs and targets are encoded with the
    statistics stored in its weights file, so the file format and the gate's
    decoding are unchanged), with a fresh Adam state and a cosine learning
    rate from `lr` to `lr_end`; each member on its own random share `bag` of
    the pairs."""
    torch = _torch()
    s0 = ens.s
    xs, ys = [], []
    for f in fields:
        rY, T, dy, _ = label_pairs(reactor, f)
        nc = T.shape[0]
        xs.append(s0.features(reactor, rY, T, f.dt, (nc + 127) // 128 * 128)[:nc])
        ys.append(s0.encode(dy))
    x, y = torch.cat(xs), torch.cat(ys)
    del xs, ys
    w = torch.ones(s0.nout, device=s0.device)
    w[0] = float(t_weight if t_weight is not None else s0.N)
    S = x.shape[0]
    for mbr, s in enumerate(ens.members):
        s._adam = None
        gen = torch.Generator(device=s.device).manual_seed(2000 + seed + mbr)
        sub = torch.randperm(S, device=s.device, generator=gen)[: int(bag * S)]
        hist = s.train(x[sub], y[sub], steps=steps, batch=batch, lr=lr, lr_end=lr_end, weights=w,
                       seed=seed + 7 * mbr, log_every=max(1, steps // 4))
        if log:
            log(f"member {mbr}: loss {[round(h[1], 5) for h in hist]}")
    return ens


class HybridReactor:
    """Surrogate-first reaction advance with gated fallback to the BDF: one
    library call (b200chem_react_hybrid) per react."""

    def __init__(self, reactor, ensemble: Ensemble, opts: HybridOpts | None = None):
        self.r = reactor
        self.ens = ensemble
        self.opts = opts or ensemble.opts
        self._sur = None
        self.last = {}

    def _handle(self):
        if self._sur is None:
            blob = self.ens.to_bytes()
            buf = ctypes.create_string_buffer(blob, len(blob))
            L = _lib.load()
            h = L.b200chem_surrogate_load(self.r._h, buf, len(blob))
            if not h:
                raise _lib.B200ChemError(-1, L.b200chem_last_error().decode())
            self._sur = h
        return self._sur

    def close(self):
        if self._sur is not None:
            _lib.load().b200chem_surrogate_destroy(self._sur)
            self._sur = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def react_flat(self, rhoY, extF_rhoY, T, rhoH, extF_rhoH, fctCount=None, mask=None, dt_react=1e-6,
                   time=0.0, stream=None, status=None, stats=True, raise_on_failure=True):
        from .reactor import ReactorError, _stream_ptr
        sur = self._handle()
        nc = T.shape[0]
        dtp = ctypes.c_double(dt_react)
        tp = ctypes.c_double(time)
        st = _lib.Stats()
        hs = _lib.HybridStats()
        o = self.opts.ctypes()
        code = _lib.load().b200chem_react_hybrid(
            self.r._h, sur, ctypes.byref(o), rhoY.data_ptr(), extF_rhoY.data_ptr(), T.data_ptr(), rhoH.data_ptr(),
            extF_rhoH.data_ptr(), fctCount.data_ptr() if fctCount is not None else None,
            mask.data_ptr() if mask is not None else None, nc, ctypes.byref(dtp), ctypes.byref(tp),
            _stream_ptr(stream), status.data_ptr() if status is not None else None,
            ctypes.byref(st) if stats else None, ctypes.byref(hs) if stats else None)
        if code != 0 and (code != -4 or raise_on_failure):
            raise ReactorError(f"hybrid react failed ({code}): {_lib.load().b200chem_last_error().decode()}")
        if stats:
            h = hs.as_dict()
            self.last = dict(h, cells=nc, accepted_fraction=h["accepted"] / max(1, h["predicted"]),
                             stats=st.as_dict())
        return dtp.value, tp.value
