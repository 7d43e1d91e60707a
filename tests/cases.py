"""Shared builders: the golden RMC problems as oracle and device objects."""
from __future__ import annotations

import types

import numpy as np

from conftest import golden


def trace_inputs(name):
    g = golden(name)
    d = {k: g[k] for k in g.files}
    d["nsp"] = d["f"].shape[0]
    return d


def ms_classes_paths(d, nsp):
    """Path classes and supercell paths of a trace (fcc, half length 5.5 A)."""
    from chimera_b200 import mspaths as MP
    cls = MP.enumerate_classes(3.59, 5.5)
    paths = MP.SupercellPaths(cls, d["ideal"], d["H"], 3.59, nsp)
    return cls, paths


def ms_table(paths, nk, seed):
    return np.random.default_rng(int(seed)).normal(0, 0.01, (paths.nent, nk))


def oracle_problem(d):
    from oracle import sampler as OS
    nsp = d["nsp"]
    nchan = d["ft_idx"].shape[0]
    nkw = nchan // nsp
    chans = [OS.Channel(d["ft_idx"][c], d["ft_frac"][c], d["ft_inside"][c], d["ft_w"][c], 2048,
                        float(d["ft_norm"]), c // nkw) for c in range(nchan)]
    ms = None
    if "ms_table_seed" in d:
        _, paths = ms_classes_paths(d, nsp)
        ms = dict(p_abs=paths.p_abs, p_cls=paths.p_cls, p_slot=paths.p_slot, inc=paths.inc,
                  cls_off=paths.cls_off, nblk=paths.nblk,
                  T=ms_table(paths, d["k"].size, d["ms_table_seed"]))
    etab, eb = None, 0.0
    if int(d.get("energy", 0)):
        V = d["V"]
        nshell = int(d["shell"].max()) + 1
        tab = np.zeros((nshell, nsp * nsp))
        m = min(nshell, V.shape[0])
        tab[:m] = 0.5 * V[:m].reshape(m, nsp * nsp)
        etab = tab.reshape(-1)
        eb = 1.0 / (8.617333262e-5 * float(d["T_ann"]))
    return OS.Problem(d["ideal"], d["i"], d["j"], d["shift"], d["shell"], d["sig2"], d["k"],
                      d["f"], d["delta"], d["lam"], float(d["s02"]), chans, d["target"],
                      d["mask"], d["sigR"], nsp, ms=ms, etab=etab, energy_beta=eb)


def device_objects(d, precision=0, reproduce=True, use_table=True):
    """(RMCSampler, ForwardModel) on the device for a golden trace."""
    from chimera_b200.forward import ForwardModel
    from chimera_b200.fourier import FourierTransform
    from chimera_b200.fourier import EdgeTransforms
    from chimera_b200.sampler import RMCSampler
    from chimera_b200.tables import ScatteringTables
    from chimera_b200 import mspaths as MP
    nsp = d["nsp"]
    cell = types.SimpleNamespace(ideal=d["ideal"], natoms=d["ideal"].shape[0], H=d["H"])
    tabs = ScatteringTables(k=d["k"], f=d["f"], delta=d["delta"], lam=d["lam"],
                            s02=float(d["s02"]))
    fm = ForwardModel(cell, tabs, d["i"], d["j"], d["shift"], sigma2=d["sig2"], shell=d["shell"])
    nchan = d["ft_idx"].shape[0]
    nkw = nchan // nsp
    per_edge = [[] for _ in range(nsp)]
    for c in range(nchan):
        f = FourierTransform(d["ft_kmodel"][c], 3.0, 13.0, (1, 2, 3)[c % nkw])
        assert np.array_equal(f._idx, d["ft_idx"][c]) and np.array_equal(f._frac, d["ft_frac"][c])
        assert np.array_equal(f._w, d["ft_w"][c])
        per_edge[c // nkw].append(f)
    ft = EdgeTransforms(per_edge)
    ms = None
    if "ms_table_seed" in d:
        _, paths = ms_classes_paths(d, nsp)
        ms = MP.SupercellMS(paths, ms_table(paths, d["k"].size, d["ms_table_seed"]))
    ep = (d["V"], float(d["T_ann"])) if int(d.get("energy", 0)) else None
    smp = RMCSampler(fm, ft, d["target"], d["mask"], d["sigR"], nrep=int(d["nrep"]),
                     tmin=float(d["tmin"]), tmax=float(d["tmax"]), seed=int(d["seed"]),
                     swap_frac=float(d["swap_frac"]), max_disp=0.10, disp_sigma=0.012,
                     energy_prior=ep, ms_library=ms, precision=precision, reproduce=reproduce,
                     use_table=use_table)
    return smp, fm
