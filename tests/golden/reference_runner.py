"""Run the converted reference (baseline/_ref) on a synthetic Hamiltonian.

Test infrastructure only (never imported by the product): it drives the
reference exactly as examples/examples_basics/main_qbasic.py does -- an NQt
one-site initialisation sweep from the occupation product state, ``fmpsQt``,
then a Qt two-site run -- with h5py/mpi4py replaced by the size-1 shims in
``tests/golden/shims``.  Hooks on ``mpo_dmrg_kernel.HVec/HDiag/renorm`` record
kernel inputs and outputs at chosen (sweep, direction, site) points.
"""
import os
import sys
import tempfile

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(HERE, "shims"))
sys.path.insert(1, os.path.join(REPO, "baseline", "_ref"))
sys.path.insert(2, REPO)

# NumPy 2 removed these aliases that the reference uses (sysutil_include.py:20, molinfo.py:58)
numpy.float_ = numpy.float64
numpy.complex_ = numpy.complex128
numpy.int = int
# The reference keys dictionaries and sorts MPO bonds by str() of lists/arrays of
# floats (qtensor_util.py:37, qtensor_opers.py:53, mpo_dmrg_dotutil.py:106);
# NumPy 1.13-style printing reproduces the formatting of its era.
numpy.set_printoptions(legacy="1.13")

import h5py  # noqa: E402  (the shim)

from qcmpodmrg_b200.hamiltonian import make_hamiltonian  # noqa: E402


def _ref():
    from qcmpodmrg.source import mpo_dmrg_class, mpo_dmrg_schedule, mpo_dmrg_kernel
    from qcmpodmrg.source.qtensor import qtensor_api, qtensor
    from qcmpodmrg.source.itools.molinfo import class_molinfo
    return mpo_dmrg_class, mpo_dmrg_schedule, mpo_dmrg_kernel, qtensor_api, qtensor, class_molinfo


def write_mole(path, ham):
    f = h5py.File(path, "w")
    cal = f.create_dataset("cal", (1,), dtype="i")
    cal.attrs["nelec"] = ham.nelec
    cal.attrs["sbas"] = ham.sbas
    cal.attrs["enuc"] = 0.0
    cal.attrs["escf"] = 0.0
    cal.attrs["ecor"] = 0.0
    f["occun"] = ham.occun
    f["orbsym"] = numpy.zeros(ham.sbas, dtype=numpy.int64)
    f["spinsym"] = numpy.array([0, 1] * (ham.sbas // 2))
    f["int1e"] = ham.int1e
    f["int2e"] = ham.int2e
    f.close()


def qt_to_dict(qt):
    """Essential fields of a reference qtensor (everything else derives from them)."""
    d = {"rank": int(qt.rank), "status": numpy.array(qt.status, dtype=bool),
         "value": numpy.array(qt.value, dtype=numpy.float64)}
    for i in range(qt.rank):
        d["qsyms%d" % i] = numpy.array(qt.qsyms[i], dtype=numpy.float64)
        d["ndims%d" % i] = numpy.array(qt.ndims[i], dtype=numpy.int64)
    if qt.idlst is not None:
        for i in range(qt.rank):
            d["idlst%d" % i] = numpy.concatenate([numpy.array(x, dtype=numpy.int64) for x in qt.idlst[i]])
    return d


class Recorder(object):
    def __init__(self, targets):
        self.targets = set(targets)   # {(isweep, status, isite)}
        self.records = {}
        self.sweep_log = []

    def key(self, dmrg, status, isite):
        return (dmrg.isweep, status, isite)


def run_reference(K, N, D, nsweeps, seed, decay=None, D0=5, targets=(), noise=0.0,
                  tol=1.e-7, maxslc=1, record_envs=True, workdir=None, npts=None, sval=0.0, sz=0.0,
                  quad="GaussLegendre", gpu=None):
    """Run the reference flow; return (result dict, recorder).

    npts: spin projection (SP-MPS) with ``npts`` quadrature points for <S^2> = sval(sval+1),
    Sz = sz, set as examples/examples_spmpsQt/main_spmps.py does (ifs2proj, s2quad); quad
    selects the reference's quadrature rule (GaussLegendre or Simpson).
    gpu: a factory init_mps -> qcmpodmrg_b200.dmrg.DMRG.  The reference's own sweep then runs
    with its kernel dispatcher patched as INTEGRATION.md shows (HVec / HDiag / renorm of the
    Qt two-site dot to qcmpodmrg_b200.mpo_dmrg_kernel, dmrg.gpu the device object); its
    Davidson, decimation, site updates and schedule stay the reference's.
    """
    mpo_dmrg_class, mpo_dmrg_schedule, mpo_dmrg_kernel, qtensor_api, qtensor, class_molinfo = _ref()
    from qcmpodmrg.source import mpo_dmrg_io
    ham = make_hamiltonian(K, N, seed, decay)
    wd = workdir or tempfile.mkdtemp(prefix="qcref_")
    cwd = os.getcwd()
    os.chdir(wd)
    rec = Recorder(targets)
    orig = (mpo_dmrg_kernel.HVec, mpo_dmrg_kernel.HDiag, mpo_dmrg_kernel.renorm,
            mpo_dmrg_kernel.SVec, mpo_dmrg_kernel.SDiag, mpo_dmrg_kernel.pRDM)
    try:
        write_mole(os.path.join(wd, "mole.h5"), ham)
        mol = class_molinfo()
        mol.comm = __import__("mpi4py").MPI.COMM_WORLD
        mol.loadHam(os.path.join(wd, "mole.h5"))
        mol.tmpdir = wd + "/"
        mol.build()
        # 0. NQt initialisation (one-site L sweep at D0) -- main_qbasic.py:36-58
        dmrg = mpo_dmrg_class.mpo_dmrg()
        dmrg.occun = mol.orboccun
        dmrg.comm = mol.comm
        dmrg.path = mol.path
        dmrg.nsite = mol.sbas // 2
        dmrg.sbas = mol.sbas
        dmrg.isym = 2
        dmrg.build()
        dmrg.qsectors = {str([float(mol.nelec), 0.0]): 1}
        dmrg.ifdvdnz = False
        sc = mpo_dmrg_schedule.schedule()
        sc.fixed(maxM=D0, maxiter=0, noise=0.0)
        dmrg.partition()
        dmrg.loadInts(mol)
        dmrg.dumpMPO()
        dmrg.default(sc)
        flmps0 = h5py.File(dmrg.path + "/lmps", "r")
        flmps1 = h5py.File(dmrg.path + "/lmpsQt", "w")
        qtensor_api.fmpsQt(flmps0, flmps1, "L")
        # record the Qt L-MPS the Qt run starts from
        init_mps = {"nsite": dmrg.nsite}
        for i in range(dmrg.nsite + 1):
            init_mps["qnum%d" % i] = numpy.array(flmps1["qnum%d" % i].value, dtype=numpy.float64)
        for i in range(dmrg.nsite):
            site = mpo_dmrg_io.loadSite(flmps1, i, True)
            init_mps["site%d" % i] = site.toDenseTensor(site.idlst)
        # 1. Qt two-site run -- main_qbasic.py:72-94
        dmrg2 = mpo_dmrg_class.mpo_dmrg()
        dmrg2.comm = mol.comm
        dmrg2.nsite = mol.sbas // 2
        dmrg2.sbas = mol.sbas
        dmrg2.isym = 2
        dmrg2.build()
        dmrg2.qsectors = {str([float(mol.nelec), 0.0]): 1}
        dmrg2.ifdvdnz = False
        sc2 = mpo_dmrg_schedule.schedule()
        sc2.fixed(ncsite=2, maxM=D, maxiter=nsweeps, tol=tol, noise=noise)
        if npts is not None:
            dmrg2.ifs2proj = True
            dmrg2.npts = npts
            dmrg2.quad = quad
            dmrg2.s2quad(sval, sz)
        mol.build()
        dmrg2.path = mol.path
        dmrg2.partition()
        dmrg2.ifQt = True
        dmrg2.ifguess = True
        dmrg2.ifprecond = True
        dmrg2.maxslc = maxslc
        dmrg2.loadInts(mol)
        dmrg2.dumpMPO()

        base = orig
        if gpu is not None:
            from qcmpodmrg_b200 import mpo_dmrg_kernel as _gpu
            dmrg2.gpu = gpu(init_mps)

            def _on_gpu(d, ncsite):
                return getattr(d, "gpu", None) is not None and d.ifQt and ncsite == 2

            def d_hvec(vec0, info, ndim0, prjmap):
                if _on_gpu(info[0], info[2]):
                    return _gpu.HVec(vec0, [info[0].gpu] + list(info[1:]), ndim0, prjmap)
                return orig[0](vec0, info, ndim0, prjmap)

            def d_hdiag(info, ndim0, prjmap):
                if _on_gpu(info[0], info[2]):
                    return _gpu.HDiag([info[0].gpu] + list(info[1:]), ndim0, prjmap)
                return orig[1](info, ndim0, prjmap)

            def d_renorm(d, isite, ncsite, flst, flstN, site, status):
                if _on_gpu(d, ncsite):
                    return _gpu.renorm(d.gpu, isite, ncsite, flst, flstN, site, status)
                return orig[2](d, isite, ncsite, flst, flstN, site, status)

            base = (d_hvec, d_hdiag, d_renorm) + tuple(orig[3:])

        def hvec_hook(vec0, info, ndim0, prjmap):
            out = base[0](vec0, info, ndim0, prjmap)
            d, isite, ncsite, flst, status, ifsym = info
            k = (d.isweep, status, isite)
            r = rec.records.setdefault(k, {})
            if k in rec.targets and "hvec_x" not in r:
                r["hvec_x"] = numpy.array(vec0)
                r["hvec_y"] = numpy.array(out)
                r["ndim0"] = ndim0
                r["prjmap"] = numpy.array(prjmap)
                r["qtmp"] = qt_to_dict(d.qtmp)
                r["qkey"] = numpy.array(d.qkey)
                r["dims"] = numpy.array(d.dims)
                if record_envs:
                    fL, fR = flst[0][0:2]
                    r["envL"] = _load_envs(qtensor, fL, d.nops)
                    r["envR"] = _load_envs(qtensor, fR, d.nops)
                    r["mpo_i"] = _load_mpo(qtensor, d.fhop, isite, d.nops)
                    r["mpo_j"] = _load_mpo(qtensor, d.fhop, isite + 1, d.nops)
                r["hpwts"] = numpy.array(d.hpwts)
                r["opers"] = numpy.array([o[0] for o in d.opers])
                if npts is not None:
                    r["opers_ipt"] = numpy.array([o[1] for o in d.opers])
                    r["qpts"] = numpy.array(d.qpts, dtype=numpy.float64)
                    r["qwts"] = numpy.array(d.qwts, dtype=numpy.float64)
            return out

        def svec_hook(vec0, info, ndim0, prjmap):
            out = orig[3](vec0, info, ndim0, prjmap)
            d, isite, ncsite, flst, status, ifsym = info
            k = (d.isweep, status, isite)
            r = rec.records.setdefault(k, {})
            if k in rec.targets and "svec_x" not in r:
                r["svec_x"] = numpy.array(vec0)
                r["svec_y"] = numpy.array(out)
                # the two-site sweep never calls SDiag (only PT does): record it on the same dot
                r["sdiag"] = numpy.array(orig[4](info, ndim0, prjmap))
                if record_envs:
                    fLp, fRp = flst[0][2:4]
                    r["penvL"] = [qt_to_dict(_load_qt(qtensor, fLp, "opers%d" % i)) for i in range(d.npts)]
                    r["penvR"] = [qt_to_dict(_load_qt(qtensor, fRp, "opers%d" % i)) for i in range(d.npts)]
                    r["pop"] = [qt_to_dict(_load_qt(qtensor, d.fpop, "op%d" % i)) for i in range(d.npts)]
            return out

        def sdiag_hook(info, ndim0, prjmap):
            out = orig[4](info, ndim0, prjmap)
            d, isite, ncsite, flst, status, ifsym = info
            k = (d.isweep, status, isite)
            r = rec.records.setdefault(k, {})
            if k in rec.targets and "sdiag" not in r:
                r["sdiag"] = numpy.array(out)
            return out

        def hdiag_hook(info, ndim0, prjmap):
            out = base[1](info, ndim0, prjmap)
            d, isite, ncsite, flst, status, ifsym = info
            k = (d.isweep, status, isite)
            r = rec.records.setdefault(k, {})
            if k in rec.targets and "hdiag" not in r:
                r["hdiag"] = numpy.array(out)
            return out

        def renorm_hook(d, isite, ncsite, flst, flstN, site, status):
            out = base[2](d, isite, ncsite, flst, flstN, site, status)
            if gpu is not None:
                return out
            k = (d.isweep, status, isite)
            r = rec.records.setdefault(k, {})
            if k in rec.targets and "renorm_site" not in r:
                r["renorm_site"] = qt_to_dict(site)
                if record_envs:
                    r["renorm_out"] = _load_envs(qtensor, flstN[0][0], d.nops)
                    if npts is not None:
                        r["renorm_pout"] = [qt_to_dict(_load_qt(qtensor, flstN[0][1], "opers%d" % i))
                                            for i in range(d.npts)]
            return out

        mpo_dmrg_kernel.HVec = hvec_hook
        mpo_dmrg_kernel.HDiag = hdiag_hook
        mpo_dmrg_kernel.renorm = renorm_hook
        mpo_dmrg_kernel.SVec = svec_hook
        mpo_dmrg_kernel.SDiag = sdiag_hook

        def prdm_hook(cimat, info):
            out = orig[5](cimat, info)
            d, isite, ncsite, flst, status, ifsym = info
            k = (d.isweep, status, isite)
            r = rec.records.setdefault(k, {})
            if k in rec.targets and "prdm_out" not in r:
                r["prdm_cimat"] = numpy.array(cimat)
                r["prdm_out"] = numpy.array(out)
                r["noise"] = float(d.noise)
            return out

        mpo_dmrg_kernel.pRDM = prdm_hook
        dmrg2.default(sc2, flmps1)
        result = {
            "K": K, "N": N, "D": D, "seed": seed, "decay": decay, "nsweeps": nsweeps,
            "eav": numpy.array(dmrg2.eav), "dwt": numpy.array(dmrg2.dwt),
            "esweeps": numpy.array([numpy.array(e).ravel()[0] for e in dmrg2.esweeps]),
            "nmvp": numpy.array(dmrg2.nmvp),
            "init_mps": init_mps,
        }
    finally:
        (mpo_dmrg_kernel.HVec, mpo_dmrg_kernel.HDiag, mpo_dmrg_kernel.renorm,
         mpo_dmrg_kernel.SVec, mpo_dmrg_kernel.SDiag, mpo_dmrg_kernel.pRDM) = orig
        os.chdir(cwd)
    return result, rec


def _load_envs(qtensor, f, nops):
    out = []
    for iop in range(nops):
        q = qtensor.Qt()
        q.load(f, "opers%d" % iop)
        assert q.nslc == 1, "fixtures assume maxslc=1"
        out.append(qt_to_dict(q.dic[0]))
    return out


def _load_qt(qtensor, f, name):
    q = qtensor.qtensor()
    q.load(f, name)
    return q


def _load_mpo(qtensor, fhop, isite, nops):
    out = []
    for iop in range(nops):
        q = qtensor.Qt()
        q.load(fhop, "site%d/op%d" % (isite, iop))
        assert q.nslc == 1
        out.append(qt_to_dict(q.dic[0]))
    return out
