"""One transform per (edge, k weight) channel (chimera/multift.py:25-84).

Same constructor and attributes as the reference adapter (fts, chi_extra,
R, nchan, chan_edge, nsp, kmin, kmax, kweights, kweight, xp); `to_R` runs
each channel's device transform. The samplers read the per-channel set-up
(`fts[c]._idx/_frac/_inside/_w/_norm/nfft`) directly and evaluate only the
fit window inside their fused step.
"""
from __future__ import annotations

import numpy as np


class MultiEdgeFT:
    def __init__(self, fts, chi_extra=None, chan_edge=None):
        self.fts = list(fts)
        self.chi_extra = None if chi_extra is None else np.ascontiguousarray(chi_extra,
                                                                             np.float64)
        R = np.asarray(self.fts[0].R)
        for f in self.fts[1:]:
            assert np.allclose(f.R, R), "channels must share the R grid"
        self.R = R
        self.nchan = len(self.fts)
        self.chan_edge = (np.arange(self.nchan, dtype=np.int32) if chan_edge is None
                          else np.asarray(chan_edge, np.int32))
        assert self.chan_edge.shape == (self.nchan,)
        self.nsp = int(self.chan_edge.max()) + 1
        self.kmin = min(f.kmin for f in self.fts)
        self.kmax = max(f.kmax for f in self.fts)
        self.kweights = tuple(dict.fromkeys(f.kweight for f in self.fts))
        self.kweight = self.fts[0].kweight
        self.xp = self.fts[0].xp

    @classmethod
    def from_spectrum(cls, S):
        return cls(S.ft, chi_extra=getattr(S, "chi_ms", None),
                   chan_edge=getattr(S, "chan_edge", None))

    def to_R(self, chi, bins=None):
        """chi (..., nsp, nk) -> complex (..., nchan, nbins)."""
        import torch
        if self.chi_extra is not None:
            extra = self.chi_extra if not isinstance(chi, torch.Tensor) else \
                torch.as_tensor(self.chi_extra, device=chi.device)
            chi = chi + extra
        out = [f.to_R(chi[..., e, :], bins=bins) for f, e in zip(self.fts, self.chan_edge)]
        if isinstance(out[0], np.ndarray):
            return np.stack(out, axis=-2)
        return torch.stack(out, dim=-2)

    def magnitude(self, chi):
        z = self.to_R(chi)
        return np.abs(z) if isinstance(z, np.ndarray) else z.abs()

    def window_mask(self, rmin, rmax):
        return (self.R >= rmin) & (self.R <= rmax)

    def n_independent(self, rmin, rmax):
        return 2 * (self.kmax - self.kmin) * (rmax - rmin) / np.pi + 2
