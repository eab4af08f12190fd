"""Simulation output and checkpoints in the reference's HDF5 layout.

``save(sim, path)`` writes what the reference's ``save()`` writes
(src/molNEsim_decomp_impl.h:107-122, src/molNEsim_decomp_spin_impl.h:126-142,
src/molNEsim_impl.h:128-144, with ``save_base`` src/molNEsim.cpp:66-90):

    /G, /Sigma            green_func::print_to_file (src/greens.cpp:202-239): datasets
                          M (matsubara), GR, GL, GTV (packed blocks, flat complex128)
                          and nt, ntau, sig, nao; unrestricted runs /G/up, /G/down, ...
    /params/beta, /mu, /hmf, /params/h0, /params/filling, /tti
    /energy/kinetic, /energy/potential, /energy/nuclear   (do_energy, :131-144)
    /solve/params/{nao, dt, nt, ntau, k, BootMax, BootTol, CorrSteps, boot_conv, mode}

plus ``/solve/last_tstp``, the last completed time step, which is what makes the file
a checkpoint.  ``load(sim, path)`` restores G, Sigma and the mean field of a
simulation of the same sizes and returns that step, so ``sim.do_tstp`` continues from
``last_tstp + 1``.  The reference writes the Matsubara component as ``M`` but its
``read_from_file`` looks for ``GM`` (src/greens.cpp:207 and :290); here the reader
accepts either name, so files of both origins load.
"""
from __future__ import annotations

import numpy as np

from ._lib import LES, RET, TV, MAT
from .greens import HostGF
from .h5io import H5File, H5Writer


def _green_to(w: H5Writer, path: str, g):
    """green_func::print_to_file of a device green_func (or a HostGF)."""
    h = g.to_host() if hasattr(g, "to_host") else g
    w[path + "/M"] = h.mat.reshape(-1)
    w[path + "/GR"] = h.ret.reshape(-1)
    w[path + "/GL"] = h.les.reshape(-1)
    w[path + "/GTV"] = h.tv.reshape(-1)
    w[path + "/nt"] = np.int32(h.nt)
    w[path + "/ntau"] = np.int32(h.ntau)
    w[path + "/sig"] = np.int32(h.sig)
    w[path + "/nao"] = np.int32(h.nao)


def read_green(f: H5File, path: str) -> HostGF:
    """green_func::read_from_file (src/greens.cpp:241-307) into a HostGF."""
    nt, ntau, sig, nao = (int(f[path + "/" + k]) for k in ("nt", "ntau", "sig", "nao"))
    g = HostGF(nt, ntau, nao, sig)
    mat = f[path + "/GM"] if (path + "/GM") in f else f[path + "/M"]
    g.mat[:] = np.asarray(mat).reshape(g.mat.shape)
    g.ret[:] = np.asarray(f[path + "/GR"]).reshape(g.ret.shape)
    g.les[:] = np.asarray(f[path + "/GL"]).reshape(g.les.shape)
    g.tv[:] = np.asarray(f[path + "/GTV"]).reshape(g.tv.shape)
    return g


def _spin_sim(sim) -> bool:
    return isinstance(sim.G, (list, tuple))


def energies(sim, t_last: int):
    """do_energy (reference src/molNEsim_decomp_impl.h:131-144): kinetic
    sum(rho .* (hmf + h0)^T) and potential 2 energy_conv (restricted; summed over the spins
    without the factor 2 when unrestricted), for t = 0 .. t_last."""
    nt = sim.nt
    ekin, epot = np.zeros(nt + 1), np.zeros(nt + 1)
    spins = range(2) if _spin_sim(sim) else [None]
    for s in spins:
        G = sim.G[s] if s is not None else sim.G
        S = sim.Sigma[s] if s is not None else sim.Sigma
        hmf = (sim.hmf[s] if s is not None else sim.hmf).download((nt + 1, sim.p.nao, sim.p.nao))
        h0 = sim.p.h0_of(s) if s is not None else sim.p.h0
        gh = G.to_host()
        for t in range(t_last + 1):
            rho = gh.get_dm(t)
            ekin[t] += np.sum(rho * (hmf[t] + h0).T).real
            epot[t] += (1.0 if s is not None else 2.0) * sim.dyson.energy_conv(t, S, G)
    return ekin, epot


def save(sim, path: str, t_last: int, mode: str = "GF2", boot_max: int = 50, boot_tol: float = 1e-12):
    """Write the simulation (rows 0 .. t_last final) in the reference's layout."""
    w = H5Writer()
    N = sim.p.nao
    spin = _spin_sim(sim)
    if spin:
        for s, sn in enumerate(("up", "down")):
            _green_to(w, f"/G/{sn}", sim.G[s])
            _green_to(w, f"/Sigma/{sn}", sim.Sigma[s])
        w["/mu"] = np.asarray(sim.mu, float)
        w["/hmf"] = np.stack([sim.hmf[s].download((sim.nt + 1, N, N)) for s in range(2)])
        w["/params/h0"] = np.stack([sim.p.h0_of(0), sim.p.h0_of(1)])
        w["/params/filling"] = np.array([np.trace(sim.G[s].to_host().get_dm(0)).real for s in range(2)])
    else:
        _green_to(w, "/G", sim.G)
        _green_to(w, "/Sigma", sim.Sigma)
        w["/mu"] = np.float64(sim.mu)
        w["/hmf"] = sim.hmf.download((sim.nt + 1, N, N))
        w["/params/h0"] = sim.p.h0
        w["/params/filling"] = np.float64(np.trace(sim.G.to_host().get_dm(0)).real)
    w["/params/beta"] = np.float64(sim.beta)
    w["/tti"] = np.int32(0)
    ekin, epot = energies(sim, t_last)
    w["/energy/kinetic"] = ekin
    w["/energy/potential"] = epot
    w["/energy/nuclear"] = np.float64(0.0)
    for k, v in (("nao", np.int32(N)), ("dt", np.float64(sim.dt)), ("nt", np.int32(sim.nt)),
                 ("ntau", np.int32(sim.ntau)), ("k", np.int32(sim.k)), ("BootMax", np.int32(boot_max)),
                 ("BootTol", np.float64(boot_tol)), ("CorrSteps", np.int32(sim.corr_steps)),
                 ("boot_conv", np.int32(1 if (sim.boot_err is not None and sim.boot_err < boot_tol) else 0)),
                 ("mode", mode)):
        w["/solve/params/" + k] = v
    w["/solve/last_tstp"] = np.int32(t_last)
    w.save(path)


def load(sim, path: str) -> int:
    """Restore G, Sigma and the mean field of ``sim`` (same nt, ntau, nao) from a file
    written by ``save``; returns the last completed time step."""
    f = H5File(path)
    spin = _spin_sim(sim)
    N = sim.p.nao
    groups = [("/G/up", "/Sigma/up"), ("/G/down", "/Sigma/down")] if spin else [("/G", "/Sigma")]
    for s, (gp, sp) in enumerate(groups):
        for dev, grp in ((sim.G[s] if spin else sim.G, gp), (sim.Sigma[s] if spin else sim.Sigma, sp)):
            h = read_green(f, grp)
            if (h.nt, h.ntau, h.nao) != (sim.nt, sim.ntau, N):
                raise ValueError(f"{path}{grp}: sizes (nt, ntau, nao) = {(h.nt, h.ntau, h.nao)} do not match the "
                                 f"simulation's {(sim.nt, sim.ntau, N)}")
            dev.from_host(h)
    hmf = np.asarray(f["/hmf"])
    if spin:
        for s in range(2):
            sim.hmf[s].upload(np.ascontiguousarray(hmf[s]))
    else:
        sim.hmf.upload(np.ascontiguousarray(hmf))
    return int(f["/solve/last_tstp"]) if "/solve/last_tstp" in f else sim.nt
