"""Shared test helpers: fixture tensors -> product layouts / device tensor sets."""
import os

import numpy

import fixtures

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return fixtures.load(os.path.join(GOLDEN, name))


def layout_of(d):
    from qcmpodmrg_b200.qtensor import Layout
    r = int(d["rank"])
    return Layout(numpy.asarray(d["status"], dtype=bool), [d["qsyms%d" % i] for i in range(r)],
                  [d["ndims%d" % i] for i in range(r)])


def tensorset(dicts, device):
    from qcmpodmrg_b200.kernels import TensorSet
    return TensorSet([layout_of(d) for d in dicts], [numpy.asarray(d["value"], dtype=numpy.float64)
                                                      for d in dicts], device=device)


def record_operators(r, device, precision="f64", use_fiber=False, fuse_w=True, panel1=True):
    """SigmaOperator / DiagOperator for a recorded reference dot."""
    from qcmpodmrg_b200.kernels import SigmaOperator, DiagOperator, Workspace
    import torch
    ws = Workspace(torch.device(device))
    isite = int(r["key"][2])
    psi = layout_of(r["qtmp"])
    L, R = tensorset(r["envL"], device), tensorset(r["envR"], device)
    Wi, Wj = tensorset(r["mpo_i"], device), tensorset(r["mpo_j"], device)
    opers = [int(x) for x in numpy.atleast_1d(r["opers"])]
    hp = numpy.atleast_1d(r["hpwts"]).astype(numpy.float64)
    qkey = numpy.asarray(r["qkey"], dtype=numpy.float64)
    sig = SigmaOperator(ws, isite, psi, L, R, Wi, Wj, qkey, opers, hp, precision, use_fiber=use_fiber,
                        fuse_w=fuse_w, panel1=panel1)
    dg = DiagOperator(ws, isite, psi, L, R, Wi, Wj, qkey, opers, hp)
    return sig, dg, ws


def record_renormalizer(r, device):
    from qcmpodmrg_b200.kernels import Renormalizer, Workspace
    import torch
    ws = Workspace(torch.device(device))
    isite = int(r["key"][2])
    status = "L" if int(r["key"][1]) == 0 else "R"
    site = layout_of(r["renorm_site"])
    opers = [int(x) for x in numpy.atleast_1d(r["opers"])]
    if status == "L":
        E, W, j = tensorset(r["envL"], device), tensorset(r["mpo_i"], device), isite
    else:
        E, W, j = tensorset(r["envR"], device), tensorset(r["mpo_j"], device), isite + 1
    rn = Renormalizer(ws, j, status, site, E, W, opers)
    return rn, numpy.asarray(r["renorm_site"]["value"], dtype=numpy.float64)


def record_sp_operators(r, device, use_fiber=True, fuse_w=False, prune=True):
    """Projected H and S operators (+ diagonals) of a recorded spin-projected reference dot
    (prune: skip the block pairs that read or write the zero blocks of the reduced vector)."""
    from qcmpodmrg_b200.kernels import SigmaOperator, DiagOperator, Workspace
    from qcmpodmrg_b200.spin import ProjectedOperator, reduce_layout, reduce_map
    import torch
    ws = Workspace(torch.device(device))
    isite = int(r["key"][2])
    lay = layout_of(r["qtmp"])
    lay_n = reduce_layout(lay)
    red = reduce_map(lay, lay_n)
    qkey = numpy.asarray(r["qkey"], dtype=numpy.float64)
    opers = [int(x) for x in numpy.atleast_1d(r["opers"])]
    hp = numpy.atleast_1d(r["hpwts"]).astype(numpy.float64)
    L, R = tensorset(r["envL"], device), tensorset(r["envR"], device)
    Wi, Wj = tensorset(r["mpo_i"], device), tensorset(r["mpo_j"], device)
    PL, PR, P = tensorset(r["penvL"], device), tensorset(r["penvR"], device), tensorset(r["pop"], device)
    qw = numpy.atleast_1d(r["qwts"]).astype(numpy.float64)
    popers = [0] * len(qw)
    opts = {"use_fiber": use_fiber, "fuse_w": fuse_w, "live": lay.allowed.astype(bool) if prune else None}
    sig = ProjectedOperator(ws, SigmaOperator(ws, isite, lay_n, L, R, Wi, Wj, qkey[:1], opers, hp, **opts), red)
    sv = ProjectedOperator(ws, SigmaOperator(ws, isite, lay_n, PL, PR, P, P, qkey[:1], popers, qw, **opts), red)
    dg = DiagOperator(ws, isite, lay, L, R, Wi, Wj, qkey, opers, hp)
    sd = DiagOperator(ws, isite, lay, PL, PR, P, P, qkey, popers, qw)
    return sig, sv, dg, sd, ws


def record_sp_renormalizers(r, device):
    """Renormalizers of the H and projector environments for a recorded SP dot, and the
    N-reduced site values they take."""
    from qcmpodmrg_b200.kernels import Renormalizer, Workspace
    from qcmpodmrg_b200.spin import reduce_layout, reduce_map
    import torch
    ws = Workspace(torch.device(device))
    isite = int(r["key"][2])
    status = "L" if int(r["key"][1]) == 0 else "R"
    site = layout_of(r["renorm_site"])
    site_n = reduce_layout(site)
    vals = numpy.zeros(site_n.size)
    vals[reduce_map(site, site_n)] = numpy.asarray(r["renorm_site"]["value"], dtype=numpy.float64)
    opers = [int(x) for x in numpy.atleast_1d(r["opers"])]
    P = tensorset(r["pop"], device)
    popers = [0] * len(r["pop"])
    if status == "L":
        E, PE, W, j = tensorset(r["envL"], device), tensorset(r["penvL"], device), tensorset(r["mpo_i"], device), isite
    else:
        E, PE, W, j = (tensorset(r["envR"], device), tensorset(r["penvR"], device), tensorset(r["mpo_j"], device),
                       isite + 1)
    rn = Renormalizer(ws, j, status, site_n, E, W, opers)
    rp = Renormalizer(ws, j, status, site_n, PE, P, popers)
    return rn, rp, vals


def _dense_qnums(qsyms, env, index):
    """Dense per-state quantum numbers of an environment index from the sector list
    ``qsyms`` (same sector order) and the environment's recorded positions (idlst)."""
    nd = numpy.asarray(env["ndims%d" % index], dtype=numpy.int64)
    pos = numpy.asarray(env["idlst%d" % index], dtype=numpy.int64)
    q = numpy.asarray(qsyms, dtype=numpy.float64).reshape(len(nd), -1)
    out = numpy.zeros((int(nd.sum()), q.shape[1]))
    out[pos] = numpy.repeat(q, nd, axis=0)
    return out


def record_noise(r, device):
    """(NoiseRDM, packed rank-3 wavefunction values, C C^T) for a recorded pRDM call;
    spin-projected records (with a quadrature) get the N-reduced layout."""
    from qcmpodmrg_b200.kernels import NoiseRDM, Workspace, scatter
    from qcmpodmrg_b200.dmrg import noise_psi_layout
    from qcmpodmrg_b200.spin import reduce_layout, reduce_map
    import torch
    ws = Workspace(torch.device(device))
    isite = int(r["key"][2])
    status = "L" if int(r["key"][1]) == 0 else "R"
    qkey = numpy.asarray(r["qkey"], dtype=numpy.float64)
    q = r["qtmp"]
    ql = _dense_qnums(q["qsyms0"], r["envL"][0], 1)
    qr = qkey - _dense_qnums(q["qsyms3"], r["envR"][0], 1)
    lay, idl, dense_idl = noise_psi_layout(ql, qr, qkey, status)
    c = numpy.asarray(r["prdm_cimat"], dtype=numpy.float64)
    vals = torch.from_numpy(c[0].reshape(-1)[lay.prjmap(idl)].copy()).to(device)
    sp = "qwts" in r
    if sp:
        lay_n = reduce_layout(lay)
        out = torch.empty(lay_n.size, dtype=torch.float64, device=device)
        vals = scatter(vals, torch.from_numpy(reduce_map(lay, lay_n)).to(device), out)
        lay, qkey = lay_n, qkey[:1]
    opers = [int(x) for x in numpy.atleast_1d(r["opers"])]
    if status == "L":
        E, W, j = tensorset(r["envL"], device), tensorset(r["mpo_i"], device), isite
        m = c.reshape(c.shape[0], c.shape[1] * c.shape[2], -1)
        cc = sum(m[i] @ m[i].T for i in range(len(m)))
    else:
        E, W, j = tensorset(r["envR"], device), tensorset(r["mpo_j"], device), isite + 1
        m = c.reshape(c.shape[0], c.shape[1], -1)
        cc = sum(m[i].T @ m[i] for i in range(len(m)))
    return NoiseRDM(ws, j, status, lay, E, W, opers, qkey, dense_idl), vals, cc


def fci_spin_states(ham, nstates=8):
    """Lowest eigenvalues of H among determinants with N//2 alpha electrons (Sz = 0, or
    -1/2 for odd N) with <S- S+> (= S(S+1) - Sz^2 - Sz), by exact diagonalisation (small
    K only): an independent check of spin-projected results."""
    from itertools import combinations
    from qcmpodmrg_b200.hamiltonian import fci_hamiltonian
    n, N = ham.sbas, ham.nelec
    na = N // 2
    alpha, beta = [2 * i for i in range(n // 2)], [2 * i + 1 for i in range(n // 2)]
    h, dets = fci_hamiltonian(ham)
    up = {d: i for i, d in enumerate(tuple(sorted(a + b)) for a in combinations(alpha, na + 1)
                                     for b in combinations(beta, N - na - 1))}
    sp = numpy.zeros((len(up), len(dets)))
    for j, d in enumerate(dets):
        for i in range(n // 2):
            a, b = 2 * i, 2 * i + 1
            if b in d and a not in d:
                occ = list(d)
                sign = (-1) ** occ.index(b)
                occ.remove(b)
                sign *= (-1) ** sum(1 for o in occ if o < a)
                sp[up[tuple(sorted(occ + [a]))], j] += sign
    w, v = numpy.linalg.eigh(h)
    s2 = numpy.einsum("ij,ik,kj->j", v, sp.T @ sp, v)
    return w[:nstates], s2[:nstates]
