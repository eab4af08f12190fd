"""Analytic 2x2 fixtures of the reference tests (tests/set_up_g.h:13-242).

``set_up_G_herm`` and ``set_up_G`` fill Green's functions and self-energies
with closed-form functions of the time indices and of the collocation points
tau = beta*(x_i+1)/2, exactly as the reference test helpers do.
"""
import numpy as np

from nedyson_b200.greens import HostGF


def _taus(x, beta):
    return beta * (np.asarray(x) + 1.0) / 2.0


def set_up_G_herm(x, G: HostGF, S: HostGF, dt, beta):
    """tests/set_up_g.h:13-109"""
    Nt, Ntau = G.nt, G.ntau
    ci = 1j
    for t in range(Nt + 1):
        for tp in range(t + 1):
            dt2 = dt * dt
            b = S.retblk(t, tp).reshape(-1)
            b[0] = ci * (dt2 * dt2 * t * t * tp * tp)
            b[1] = ci * (dt2 * t * tp)
            b[2] = ci * (dt2 * t * tp)
            dt3 = dt2 * dt
            b[3] = ci * (dt3 * dt3 * t ** 3 * tp ** 3)
    for tp in range(Nt + 1):
        for t in range(tp + 1):
            b = G.lesblk(t, tp).reshape(-1)
            b[0] = ci * np.exp(ci * (t - tp) * dt)
            b[1] = (t - tp) * dt
            b[2] = (t - tp) * dt
            b[3] = ci * np.exp(3. * ci * (t - tp) * dt)
    for tp in range(Nt + 1):
        for t in range(tp + 1):
            dt2 = dt * dt
            b = S.lesblk(t, tp).reshape(-1)
            b[0] = ci * (dt2 * t * tp)
            b[1] = ci * np.exp(2. * ci * (dt * (t - tp)))
            b[2] = ci * np.exp(2. * ci * (dt * (t - tp)))
            b[3] = dt * (t - tp)
    for t in range(Nt + 1):
        for tp in range(t + 1):
            b = G.retblk(t, tp).reshape(-1)
            b[0] = -ci * np.cos(3. * dt * (t - tp))
            b[1] = -np.sin(2. * dt * (t - tp))
            b[2] = -np.sin(2. * dt * (t - tp))
            b[3] = -ci * np.cos(dt * (t - tp))
    taus = _taus(x, beta)
    for t in range(Nt + 1):
        for m in range(Ntau + 1):
            tp = taus[m]
            b = G.tv[t, m].reshape(-1)
            b[0] = tp * tp
            b[1] = ci * (dt * t)
            b[2] = np.exp(ci * tp)
            b[3] = dt * dt * t * t - ci * tp
            b = S.tv[t, m].reshape(-1)
            b[0] = dt * t * tp
            b[1] = dt * dt * t * t * tp
            b[2] = np.sin(dt * t)
            b[3] = ci * (dt * t - tp)
    for m in range(Ntau + 1):
        tp = taus[m]
        b = G.mat[m].reshape(-1)
        b[0], b[1], b[2], b[3] = tp, ci * tp, tp * tp, np.exp(ci * tp)
        b = S.mat[m].reshape(-1)
        b[0], b[1], b[2], b[3] = tp * ci, tp, np.sin(tp * tp), np.exp(ci * tp)


def set_up_G(x, G: HostGF, Gcc: HostGF, S: HostGF, Scc: HostGF, dt, beta):
    """tests/set_up_g.h:115-242"""
    Nt, Ntau = G.nt, G.ntau
    Gsig, Ssig = G.sig, S.sig
    ci = 1j
    cj = np.conj
    for t in range(Nt + 1):
        for tp in range(t + 1):
            b = S.retblk(t, tp).reshape(-1)
            b[0] = dt * dt * dt * t * tp * tp
            b[1] = ci * (dt * t) - dt * tp
            b[2] = np.sin(dt * t)
            b[3] = np.cos(dt * tp)
            c = Scc.retblk(t, tp).reshape(-1)
            c[0] = -cj(dt * dt * dt * tp * t * t)
            c[2] = -cj(ci * (dt * tp) - dt * t)
            c[1] = -cj(np.sin(dt * tp))
            c[3] = -cj(np.cos(dt * t))
    for tp in range(Nt + 1):
        for t in range(tp + 1):
            b = S.lesblk(t, tp).reshape(-1)
            b[0] = dt * dt * dt * t * t * tp
            b[1] = dt * t + 2. * dt * tp
            b[2] = np.exp(ci * (dt * t))
            b[3] = np.exp(ci * (t - tp) * dt)
            c = Scc.lesblk(t, tp).reshape(-1)
            c[0] = -cj(dt * dt * dt * tp * tp * t)
            c[2] = -cj(dt * tp + 2. * dt * t)
            c[1] = -cj(np.exp(ci * (dt * tp)))
            c[3] = -cj(np.exp(ci * (tp - t) * dt))
    taus = _taus(x, beta)
    for t in range(Nt + 1):
        for m in range(Ntau + 1):
            tp = taus[m]
            b = S.tv[t, m].reshape(-1)
            b[0] = dt * t * tp
            b[1] = np.cos(dt * t * tp)
            b[2] = np.exp(ci * tp)
            b[3] = dt * t - tp
            c = Scc.tv[t, m].reshape(-1)
            c[0] = -Ssig * cj(ci - dt * t * (beta - tp))
            c[2] = -Ssig * cj(np.sin(2 * (beta - tp)))
            c[1] = -Ssig * cj(3 * (beta - tp) + dt * t)
            c[3] = -Ssig * cj(dt * t * ci)
    for m in range(Ntau + 1):
        tp = taus[m]
        b = S.mat[m].reshape(-1)
        b[0], b[1], b[2], b[3] = 1, tp, 2, ci * tp * tp
    for t in range(Nt + 1):
        for tp in range(t + 1):
            b = G.retblk(t, tp).reshape(-1)
            b[0] = dt * (t + tp)
            b[1] = dt * (t + 2 * tp)
            b[2] = dt * (t + 3 * tp)
            b[3] = ci * np.cos(dt * tp)
            c = Gcc.retblk(t, tp).reshape(-1)
            c[0] = -cj(dt * (tp + t))
            c[2] = -cj(dt * (tp + 2 * t))
            c[1] = -cj(dt * (tp + 3 * t))
            c[3] = -cj(ci * np.cos(dt * t))
    for tp in range(Nt + 1):
        for t in range(tp + 1):
            b = G.lesblk(t, tp).reshape(-1)
            b[0] = t * dt * ci
            b[1] = tp * dt * ci
            b[2] = dt * (t - tp)
            b[3] = 4
            c = Gcc.lesblk(t, tp).reshape(-1)
            c[0] = -cj(tp * dt * ci)
            c[2] = -cj(t * dt * ci)
            c[1] = -cj(dt * (tp - t))
            c[3] = -cj(4)
    for t in range(Nt + 1):
        for m in range(Ntau + 1):
            tp = taus[m]
            b = G.tv[t, m].reshape(-1)
            b[0] = dt * t
            b[1] = ci * 2.
            b[2] = tp
            b[3] = tp * tp
            c = Gcc.tv[t, m].reshape(-1)
            c[0] = -Gsig * cj(dt * t * (beta - tp))
            c[2] = -Gsig * cj(ci * (beta - tp))
            c[1] = -Gsig * cj(ci - (beta - tp))
            c[3] = -Gsig * cj(dt * t + (beta - tp))
    for m in range(Ntau + 1):
        tp = taus[m]
        b = G.mat[m].reshape(-1)
        b[0], b[1], b[2], b[3] = np.exp(ci * tp), np.exp(ci * tp), np.cos(tp), ci
