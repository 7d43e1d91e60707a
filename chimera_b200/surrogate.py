"""The swap surrogate and delayed acceptance (no reference counterpart).

A proposed swap of sites lo < hi (species p = S[lo] != q = S[hi]) is
described by the unordered pair {p, q} and the species around the two sites:
the D neighbours of each site in one translation-invariant order
(`feature_neighbours`), with code nsp where a neighbour is lo or hi itself.
Together with the chain the move belongs to (ladder and rung: the chains'
current residuals differ, and the network learns one input row per chain)
and ln(beta) of the rung this is the input of a BF16 MLP (three hidden ReLU
layers of H units, FP32 accumulation) whose output, times the orientation
sign sigma = +1 if p < q else -1 and a scale, predicts the swap's chi^2
change d. A swap and its reverse have the same input and so opposite
predictions, which is what keeps delayed acceptance exact
(Christen & Fox 2005, J. Comput. Graph. Stat. 14:795):

    stage 1  accept with min(1, exp(-beta nfit d^ - E))      (E: exact prior)
    stage 2  accept with min(1, exp(-beta nfit (d - d^)))    (exact d)

Stage 1 runs inside the fused sampler step before the exact evaluation;
only moves that pass it pay for the exact path sum, transform and chi^2.

Training uses swaps logged by the sampler itself (features and sigma * d of
every swap it evaluates exactly): the library's own kernels compute the
gradient (tensor-core GEMMs for the dense layers) and the Adam step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def feature_neighbours(ideal, iidx, jidx, shift, ncoord):
    """(natoms, ncoord) int32: each site's neighbours (the pair list's j of
    its pairs) sorted by (distance, dx, dy, dz) of the ideal displacement, the
    same order at every site of a Bravais supercell."""
    ideal = np.asarray(ideal, np.float64)
    iidx, jidx = np.asarray(iidx), np.asarray(jidx)
    natoms = ideal.shape[0]
    assert np.array_equal(iidx, np.repeat(np.arange(natoms), ncoord)), "pairs must be i-major"
    d = ideal[jidx] + np.asarray(shift, np.float64) - ideal[iidx]
    r = np.linalg.norm(d, axis=1)
    key = np.round(np.stack([r, d[:, 0], d[:, 1], d[:, 2]], 1), 6).reshape(natoms, ncoord, 4)
    J = jidx.reshape(natoms, ncoord)
    out = np.empty((natoms, ncoord), np.int32)
    for i in range(natoms):
        o = np.lexsort(key[i, :, ::-1].T)
        out[i] = J[i, o]
    return out


class SwapSurrogate:
    """Parameters, Adam state and device descriptor of one surrogate."""

    def __init__(self, nsp, D, H=256, nchain=0, seed=0):
        import torch
        N.require_cuda()
        self.torch = torch
        self.nsp, self.D, self.H, self.nchain = int(nsp), int(D), int(H), int(nchain)
        self.nin = self.nsp * (self.nsp - 1) // 2 + 2 * self.D * (self.nsp + 1) + self.nchain
        self.nparam = int(N.lib().chx_mlp_nparam(self.nsp, self.D, self.nchain, self.H))
        if self.nparam <= 0:
            raise N.ChxError(f"surrogate shape nsp={nsp} D={D} nchain={nchain} H={H} "
                             "not supported")
        self.theta = torch.zeros(self.nparam, dtype=torch.float32, device="cuda")
        self.theta16 = torch.zeros(self.nparam, dtype=torch.int16, device="cuda")
        self.m = torch.zeros_like(self.theta)
        self.v = torch.zeros_like(self.theta)
        self.grad_buf = torch.zeros_like(self.theta)
        self.t = 0
        self.host = N.Mlp()
        N.call("chx_mlp_bind", C.byref(self.host), self.nsp, self.D, self.nchain, self.H,
               N.ptr(self.theta), N.ptr(self.theta16))
        self.host.out_scale, self.host.feat_shift, self.host.feat_scale = 1.0, 0.0, 1.0
        # one device descriptor for the surrogate's life: ladders keep its address
        self.d_desc = torch.zeros(C.sizeof(N.Mlp), dtype=torch.uint8, device="cuda")
        self.init(seed)

    # ---------------------------------------------------------- layout
    def offsets(self):
        H, nin = self.H, self.nin
        o = {"W1": 0}
        o["b1"] = o["W1"] + (nin + 1) * H
        o["W2"] = o["b1"] + H
        o["b2"] = o["W2"] + H * H
        o["W3"] = o["b2"] + H
        o["b3"] = o["W3"] + H * H
        o["w4"] = o["b3"] + H
        o["b4"] = o["w4"] + H
        return o

    def set_params(self, theta):
        import torch
        th = torch.as_tensor(np.asarray(theta, np.float32)).to("cuda").contiguous()
        assert th.numel() == self.nparam
        self.theta.copy_(th)
        self.theta16.copy_(self.theta.to(torch.bfloat16).view(torch.int16))
        self.upload()

    def init(self, seed=0, zero=False):
        """He-normal weights (zero biases); zero=True gives the zero network."""
        rng = np.random.default_rng(seed)
        H, nin = self.H, self.nin
        th = np.zeros(self.nparam, np.float32)
        if not zero:
            o = self.offsets()
            fan1 = 2 * self.D + 3
            th[o["W1"]:o["b1"]] = rng.normal(0, np.sqrt(2.0 / fan1), (nin + 1) * H)
            th[o["W2"]:o["b2"]] = rng.normal(0, np.sqrt(2.0 / H), H * H)
            th[o["W3"]:o["b3"]] = rng.normal(0, np.sqrt(2.0 / H), H * H)
            th[o["w4"]:o["b4"]] = rng.normal(0, np.sqrt(1.0 / H), H)
        self.m.zero_()
        self.v.zero_()
        self.t = 0
        self.set_params(th)

    def upload(self):
        """Copy the host descriptor into the device descriptor (in stream
        order, after a scale change)."""
        raw = bytes(C.string_at(C.addressof(self.host), C.sizeof(self.host)))
        self.d_desc.copy_(self.torch.frombuffer(bytearray(raw), dtype=self.torch.uint8))
        return self.d_desc

    @property
    def device_ptr(self):
        return N.dptr(self.d_desc)

    # --------------------------------------------------------- compute
    def _chain(self, chain):
        if chain is None:
            return None
        return self.torch.as_tensor(chain).to("cuda", self.torch.int32).contiguous()

    def predict(self, codes, lnbeta, chain=None):
        """Network output (B,) for codes (B, 1 + 2D) uint8, lnbeta (B,)
        float32 and chain (B,) (or None), by the sampler's own per-CTA code
        (device tensors in and out)."""
        torch = self.torch
        codes = torch.as_tensor(codes).to("cuda", torch.uint8).contiguous()
        lnb = torch.as_tensor(lnbeta).to("cuda", torch.float32).contiguous()
        ch = self._chain(chain)
        out = torch.empty(codes.shape[0], dtype=torch.float32, device="cuda")
        N.call("chx_mlp_predict", N.ptr(self.d_desc), N.ptr(codes), N.ptr(lnb), N.ptr(ch),
               codes.shape[0], N.ptr(out), N.stream())
        return out

    def _work(self, B):
        nb = int(N.lib().chx_mlp_work_bytes(B, self.H))
        w = getattr(self, "_wk", None)
        if w is None or w.numel() < nb:
            self._wk = self.torch.empty(nb, dtype=self.torch.uint8, device="cuda")
        return self._wk

    def grad(self, codes, lnbeta, target, chain=None):
        """(loss, y, grad) of the mean squared error of the network output
        against target (normalised units) on one batch; chain, when given,
        must be sorted ascending (fit sorts each batch)."""
        torch = self.torch
        codes = torch.as_tensor(codes).to("cuda", torch.uint8).contiguous()
        lnb = torch.as_tensor(lnbeta).to("cuda", torch.float32).contiguous()
        tgt = torch.as_tensor(target).to("cuda", torch.float32).contiguous()
        B = codes.shape[0]
        ch = self._chain(chain)
        y = torch.empty(B, dtype=torch.float32, device="cuda")
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        N.call("chx_mlp_grad", C.byref(self.host), N.ptr(codes), N.ptr(lnb), N.ptr(ch),
               N.ptr(tgt), B, N.ptr(y), N.ptr(self.grad_buf), N.ptr(loss),
               N.ptr(self._work(B)), N.stream())
        return loss, y, self.grad_buf

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.t += 1
        N.call("chx_mlp_adam", N.ptr(self.theta), N.ptr(self.theta16), N.ptr(self.grad_buf),
               N.ptr(self.m), N.ptr(self.v), self.nparam, lr, beta1, beta2, eps, self.t,
               N.stream())

    def fit(self, codes, lnbeta, y, chain=None, epochs=4, batch=4096, lr=1e-3, seed=0,
            holdout=0.1):
        """Train on logged swaps: codes (n, 1 + 2D), lnbeta (n,), y = sigma * d
        (n,), chain (n,) or None. Sets the output and feature scales from the
        data, then runs Adam over shuffled batches (each sorted by chain).
        Returns {"loss": per-epoch mean training loss, "rmse_d": held-out RMS
        error of d^ in chi^2 units, "std_d": held-out sd of d, "n": n}."""
        torch = self.torch
        codes = torch.as_tensor(codes).to("cuda", torch.uint8).contiguous()
        lnb = torch.as_tensor(lnbeta).to("cuda", torch.float32).contiguous()
        y = torch.as_tensor(y).to("cuda", torch.float32).contiguous()
        n = codes.shape[0]
        ch = self._chain(chain) if self.nchain else None
        g = torch.Generator(device="cpu").manual_seed(seed)
        perm = torch.randperm(n, generator=g).to("cuda")
        nho = int(n * holdout) if n >= 20 else 0
        ho, tr = perm[:nho], perm[nho:]
        ys = float(y[tr].float().std()) if tr.numel() > 1 else 1.0
        self.host.out_scale = ys if ys > 0 else 1.0
        lb = lnb[tr]
        self.host.feat_shift = float(lb.mean())
        sd = float(lb.std()) if tr.numel() > 1 else 0.0
        self.host.feat_scale = 1.0 / sd if sd > 1e-6 else 1.0
        self.upload()
        t = y / self.host.out_scale
        hist = []
        for ep in range(epochs):
            order = tr[torch.randperm(tr.numel(), generator=g).to("cuda")]
            tot, nb = torch.zeros((), device="cuda"), 0
            for s in range(0, order.numel() - batch + 1 if order.numel() >= batch else 1, batch):
                idx = order[s:s + batch]
                cb = None
                if ch is not None:
                    cb, o = torch.sort(ch[idx], stable=True)
                    idx = idx[o]
                loss, _, _ = self.grad(codes[idx], lnb[idx], t[idx], cb)
                self.adam(lr)
                tot += loss[0]
                nb += 1
            hist.append(float(tot) / max(nb, 1))
        out = {"loss": hist, "n": n}
        if nho:
            pred = self.predict(codes[ho], lnb[ho], None if ch is None else ch[ho])
            pred = pred * self.host.out_scale
            out["rmse_d"] = float(((pred - y[ho]) ** 2).mean().sqrt())
            out["std_d"] = float(y[ho].std())
        return out
