"""Drop-in for the reference's kernel dispatch module (source/mpo_dmrg_kernel.py).

Same function names, arguments and return conventions as the functions that
mpo_dmrg_dot.ci_solver, dotutil.genHDiag and mpo_dmrg_opt.sweep call:

  HDiag(info, ndim0, prjmap)                       source/mpo_dmrg_kernel.py:41-51
  HVec(vec0, info, ndim0, prjmap)                  source/mpo_dmrg_kernel.py:117-136
  SDiag(info, ndim0, prjmap)                       source/mpo_dmrg_kernel.py:183-190
  SVec(vec0, info, ndim0, prjmap)                  source/mpo_dmrg_kernel.py:226-231
  renorm(dmrg, isite, ncsite, flst, flstN, site, status)   :347-377
  pRDM(cimat, info)                                :278-282 (with the noise term, pRDMQt)

With a spin-projected ``dmrg`` (qcmpodmrg_b200.spin.SPDMRG, the reference's
ifs2proj) HVec/HDiag are the projected Hamiltonian's, SVec/SDiag the projector's
(zero without projection, as in the reference), and renorm also renormalises the
projector's environments (renormQt_S00), stored in ``flstN[0][1]``.

``info = [dmrg, isite, ncsite, flst, status, ifsym]`` as in mpo_dmrg_dot.py:31.
Here ``dmrg`` is a qcmpodmrg_b200.dmrg.DMRG (device-resident environments);
``flst[0][0:2]`` / ``flstN[0][0]`` are the device environment sets standing in
for the reference's per-site HDF5 files.  Vectors may be NumPy arrays (host
buffers, copied to and from the device inside the call) or CUDA tensors.  Only
the two-site Qt path exists (ncsite == 2, ifQt); anything else raises.
"""
import numpy
import torch



def _check(info):
    dmrg, isite, ncsite, flst, status, ifsym = info
    if ncsite != 2:
        raise NotImplementedError("only the two-site dot is implemented")
    return dmrg, isite


def _ops(dmrg, isite):
    """Sigma/diagonal operators of the dot, cached on the DMRG object while the dot is active."""
    L, R = dmrg.lenv[isite - 1], dmrg.renv[isite + 2]
    cache = getattr(dmrg, "_dot_cache", None)
    if cache is None or cache[0] != isite or cache[1] is not L or cache[2] is not R:
        lay, idl, sig, dg = dmrg.dot_operators(isite)
        dmrg._dot_cache = (isite, L, R, lay, idl, sig, dg)      # environments held: compared by identity
    return dmrg._dot_cache[3:]


def _to_dev(v, dev):
    if torch.is_tensor(v):
        return v.to(dev, torch.float64)
    return torch.from_numpy(numpy.ascontiguousarray(v, dtype=numpy.float64)).to(dev)


def HVec(vec0, info, ndim0, prjmap, precision=None):
    """sigma = H_eff vec0 in the packed (qtmp) layout.  ``precision`` (an addition to the
    reference's signature, optional) overrides the sigma precision of the DMRG object for
    this call, e.g. "f64" for the FP64 check of a mixed-precision solve."""
    dmrg, isite = _check(info)
    lay, idl, sig, dg = _ops(dmrg, isite)
    if ndim0 != sig.ndim0:
        raise ValueError("ndim0 does not match the dot's wavefunction template")
    y = sig(_to_dev(vec0, dmrg.device), precision=precision)
    return y if torch.is_tensor(vec0) else y.cpu().numpy()


def HDiag(info, ndim0, prjmap):
    """Diagonal of H_eff in the packed layout (real)."""
    dmrg, isite = _check(info)
    lay, idl, sig, dg = _ops(dmrg, isite)
    return dg().cpu().numpy()


def _sops(dmrg, isite):
    """Projector operators of a spin-projected dot, cached like _ops."""
    PL, PR = dmrg.plenv[isite - 1], dmrg.prenv[isite + 2]
    cache = getattr(dmrg, "_sdot_cache", None)
    if cache is None or cache[0] != isite or cache[1] is not PL or cache[2] is not PR:
        sv, sd = dmrg.dot_projector(isite)
        dmrg._sdot_cache = (isite, PL, PR, sv, sd)
    return dmrg._sdot_cache[3:]


def SVec(vec0, info, ndim0, prjmap):
    """S vec0 = P vec0 with the spin projector in the packed layout (SVecQt); zero
    without spin projection."""
    dmrg, isite = _check(info)
    if not getattr(dmrg, "ifs2proj", False):
        z = numpy.zeros(ndim0)
        return torch.from_numpy(z).to(vec0.device) if torch.is_tensor(vec0) else z
    sv, sd = _sops(dmrg, isite)
    if ndim0 != sv.ndim0:
        raise ValueError("ndim0 does not match the dot's wavefunction template")
    y = sv(_to_dev(vec0, dmrg.device))
    return y if torch.is_tensor(vec0) else y.cpu().numpy()


def SDiag(info, ndim0, prjmap):
    """Diagonal of the spin projector in the packed layout (SDiagQt); zero without projection."""
    dmrg, isite = _check(info)
    if not getattr(dmrg, "ifs2proj", False):
        return numpy.zeros(ndim0)
    sv, sd = _sops(dmrg, isite)
    return sd().cpu().numpy()


class QtSite(object):
    """A site tensor handed over by the reference (its ``qtensor``: status, qsyms, ndims and
    the packed ``value`` array, source/qtensor/qtensor.py:108-149) as the device operators
    take it: the packed layout and the values on the device."""

    def __init__(self, qt, device):
        from .qtensor import Layout
        self.layout = Layout(numpy.asarray(qt.status, dtype=bool),
                             [numpy.asarray(q, dtype=numpy.float64) for q in qt.qsyms],
                             [numpy.asarray(n, dtype=numpy.int64) for n in qt.ndims])
        self.values = torch.from_numpy(numpy.ascontiguousarray(qt.value, dtype=numpy.float64)).to(device)

    def bond_qnums(self, index):
        """Per-state quantum numbers of one index, sector by sector (its classification
        returns the same sectors in the same order)."""
        q = self.layout.qsyms[index]
        n = self.layout.ndims[index]
        return numpy.repeat(numpy.asarray(q, dtype=numpy.float64).reshape(len(n), -1), n, axis=0)


def renorm(dmrg, isite, ncsite, flst, flstN, site, status):
    """New environments of every operator; stored in flstN[0][0] (when given) and in dmrg's
    env table (with spin projection also the projector's, renormQt_S00, in flstN[0][1]).

    ``site`` is a qcmpodmrg_b200.dmrg.SiteTensor (packed values on the device) or the
    reference's own qtensor site (mpo_dmrg_opt.sweep passes it, source/mpo_dmrg_opt.py:66):
    then its values are copied to the device and the new bond's quantum numbers (its right
    index for 'L', left index for 'R') become those of the next dots.
    """
    if ncsite != 2:
        raise NotImplementedError("only the two-site dot is implemented")
    j = isite if status == "L" else isite + ncsite - 1
    if not hasattr(site, "layout"):
        site = QtSite(site, dmrg.device)
        if status == "L":
            dmrg.qnuml[j + 1] = site.bond_qnums(2)
        else:
            dmrg.qnumr[j] = site.bond_qnums(0)
    dmrg.renormalize(j, status, site)
    sp = getattr(dmrg, "ifs2proj", False)
    new = dmrg.lenv[j] if status == "L" else dmrg.renv[j]
    if flstN is not None:
        if hasattr(flstN[0][0], "create_group"):
            # the reference's own environment file: the values stay on the device; the
            # block headers its dot set-up reads (genDimensions, source/mpo_dmrg_dotutil.py:60-80)
            # are written as renormQt_H00's dumpSLC would (qtensor.dump, qtensor.py:195-206)
            _write_env_headers(flstN[0][0], new)
        else:
            flstN[0][0] = new
            if sp:
                flstN[0][1] = dmrg.plenv[j] if status == "L" else dmrg.prenv[j]
    return 0


def _write_env_headers(f, tset):
    for i, lay in enumerate(tset.layouts):
        g = f.create_group("opers%d_slc0" % i)
        g.attrs["rank"] = int(lay.rank)
        g.attrs["nqnum"] = 2
        g.attrs["nsyms"] = numpy.asarray(lay.nsyms, dtype=numpy.int64)
        g.attrs["shape"] = numpy.asarray(lay.shape, dtype=numpy.int64)
        g.attrs["size"] = int(numpy.prod(lay.shape))
        g.attrs["nblks_allowed"] = int(len(lay.idx_allowed))
        g.attrs["size_allowed"] = int(lay.size)
        g.attrs["status"] = numpy.asarray(lay.status, dtype=bool)


def pRDM(cimat, info):
    """Density matrix of the kept half of the dot, sum_i C_i C_i^+, plus dmrg.noise times
    the noise term sum_p (L_p C W_p)(L_p C W_p)^+ when dmrg.noise >= 1e-10 (pRDMQt)."""
    dmrg, isite, ncsite, flst, status, ifsym = info
    if ncsite != 2:
        raise NotImplementedError("only the two-site dot is implemented")
    c = _to_dev(cimat, dmrg.device)
    neig = c.shape[0]
    if status == "L":      # cimat [neig, ldim, dim, crdim] (dotutil.py:276-281)
        ldim, rdim = c.shape[1], c.shape[3] // 4
    else:                  # cimat [neig, lcdim, dim, rdim] (dotutil.py:282-288)
        ldim, rdim = c.shape[1] // 4, c.shape[3]
    rdm = dmrg.prdm(c.reshape(neig, -1), isite, status, (ldim, 16, rdim, ldim * 16 * rdim))
    return rdm.cpu().numpy()
