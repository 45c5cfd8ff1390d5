"""MPS files in the reference's HDF5 layout (source/mpo_dmrg_io.py:100-161).

An MPS file holds ``nsite``, the bond quantum numbers ``qnum0`` .. ``qnum<nsite>`` and the
site tensors ``site0`` .. ``site<nsite-1>``: dense arrays [l, n, r] (loadMPS icase=1) or,
for symmetry-blocked runs, one group per site in qtensor.dump's layout (icase=2,
source/qtensor/qtensor.py:188-214): attributes rank, nqnum, nsyms, shape, size, nblks,
nblks_allowed, size_allowed, savings, status and the datasets iblks_allowed (flat block
index + 1 at allowed blocks, 0 elsewhere, shaped nsyms), dims_allowed (every block's
dimensions, row-major block order), idx_allowed, ndim_allowed, ioff_allowed, value (the
packed blocks), qsyms (sectors stacked), ndims (sector sizes concatenated) and idlst (each
index's sector -> dense positions, concatenated).

The functions take an open h5py-style file object (``h5py.File`` or anything with the
same group / dataset / attrs interface); this module itself imports no HDF5 library.
Datasets are read with ``ds[()]``, which both h5py 2 and 3 support.
"""
import numpy
import torch

from .qtensor import Layout


def _read(ds):
    return numpy.asarray(ds[()])


def dump_qtensor(f, name, layout, values, idlst=None):
    """Write one symmetry-blocked tensor (packed ``values`` in ``layout``) as qtensor.dump does."""
    values = values.detach().cpu().numpy() if torch.is_tensor(values) else numpy.asarray(values)
    if len(values) != layout.size:
        raise ValueError("dump_qtensor: %d values for a layout of %d" % (len(values), layout.size))
    grp = f.create_group(name)
    size = int(numpy.prod(layout.shape))
    nall = len(layout.idx_allowed)
    grp.attrs["rank"] = layout.rank
    grp.attrs["nqnum"] = layout.nqnum
    grp.attrs["nsyms"] = layout.nsyms.astype(numpy.int32)
    grp.attrs["shape"] = layout.shape.astype(numpy.int64)
    grp.attrs["size"] = size
    grp.attrs["nblks"] = layout.nblks
    grp.attrs["nblks_allowed"] = nall
    grp.attrs["size_allowed"] = layout.size
    grp.attrs["savings"] = float(layout.size) / size if size else 0.0
    grp.attrs["status"] = numpy.asarray(layout.status, dtype=bool)
    iblks = numpy.zeros(layout.nblks, dtype=numpy.int32)
    iblks[layout.idx_allowed] = layout.idx_allowed + 1
    grp["iblks_allowed"] = iblks.reshape(tuple(layout.nsyms))
    grids = numpy.meshgrid(*[numpy.asarray(n, dtype=numpy.int32) for n in layout.ndims], indexing="ij")
    dims = numpy.stack([g.ravel() for g in grids], axis=1).astype(numpy.int32)       # every block, row-major
    grp["dims_allowed"] = dims
    grp["idx_allowed"] = layout.idx_allowed.astype(numpy.int64)
    grp["ndim_allowed"] = numpy.prod(dims.astype(numpy.int64), axis=1)
    ioff = numpy.zeros(layout.nblks, dtype=numpy.int64)
    ioff[layout.idx_allowed] = layout.ioff[layout.idx_allowed]
    grp["ioff_allowed"] = ioff
    grp["value"] = values.astype(numpy.float64)
    grp["qsyms"] = numpy.vstack(layout.qsyms)
    grp["ndims"] = numpy.hstack(layout.ndims).astype(numpy.int64)
    if idlst is not None:
        grp["idlst"] = numpy.hstack([numpy.concatenate([numpy.asarray(x, dtype=numpy.int64) for x in il])
                                     for il in idlst])
    return grp


def load_qtensor(f, name):
    """Read a tensor written by qtensor.dump (or dump_qtensor): (Layout, packed values, idlst
    or None).  The layout is rebuilt from status, sectors and sector sizes and checked
    against the stored block offsets."""
    grp = f[name]
    rank = int(grp.attrs["rank"])
    nsyms = numpy.asarray(grp.attrs["nsyms"], dtype=numpy.int64)
    status = numpy.asarray(grp.attrs["status"], dtype=bool)
    qs = _read(grp["qsyms"])
    nd = _read(grp["ndims"])
    o = numpy.concatenate([[0], numpy.cumsum(nsyms)])
    qsyms = [qs[o[i]:o[i + 1]] for i in range(rank)]
    ndims = [nd[o[i]:o[i + 1]] for i in range(rank)]
    lay = Layout(status, qsyms, ndims)
    ioff = _read(grp["ioff_allowed"])
    idx = _read(grp["idx_allowed"])
    if not (numpy.array_equal(idx, lay.idx_allowed) and numpy.array_equal(ioff[idx], lay.ioff[idx])):
        raise ValueError("load_qtensor: %s: stored block offsets differ from the layout of its sectors" % name)
    values = _read(grp["value"]).astype(numpy.float64)
    idlst = None
    if "idlst" in grp:
        flat = _read(grp["idlst"]).astype(numpy.int64)
        shape = numpy.asarray(grp.attrs["shape"], dtype=numpy.int64)
        so = numpy.concatenate([[0], numpy.cumsum(shape)])
        idlst = []
        for i in range(rank):
            part = flat[so[i]:so[i + 1]]
            co = numpy.concatenate([[0], numpy.cumsum(ndims[i])])
            idlst.append([part[co[k]:co[k + 1]] for k in range(len(ndims[i]))])
    return lay, values, idlst


def save_mps(f, d, qt=True):
    """Write the left-canonical MPS of DMRG ``d`` (its site tensors and bond quantum numbers,
    as after a left-to-right sweep) in the reference's layout: qtensor groups (qt=True, what
    its symmetry-blocked runs write) or dense arrays (qt=False)."""
    for key in list(f):
        if key == "nsite" or key.startswith("site") or key.startswith("qnum"):
            del f[key]
    f["nsite"] = d.nsite
    for i in range(d.nsite + 1):
        f["qnum%d" % i] = numpy.asarray(d.qnuml[i], dtype=numpy.float64)
    for i in range(d.nsite):
        st = d.lmps[i]
        if qt:
            dump_qtensor(f, "site%d" % i, st.layout, st.values, st.idlst)
        else:
            f["site%d" % i] = st.dense.detach().cpu().numpy()
    return 0


def load_mps(f):
    """Read an MPS file in the reference's layout (dense or qtensor sites) into the start-MPS
    dictionary DMRG.load_mps / DMRG.run take: {"site<i>": dense [l, n, r], "qnum<i>": [n, 2]}."""
    nsite = int(_read(f["nsite"]))
    out = {}
    for i in range(nsite + 1):
        out["qnum%d" % i] = _read(f["qnum%d" % i]).astype(numpy.float64).reshape(-1, 2)
    for i in range(nsite):
        node = f["site%d" % i]
        if hasattr(node, "attrs") and "rank" in node.attrs:
            lay, values, idlst = load_qtensor(f, "site%d" % i)
            if idlst is None:
                raise ValueError("load_mps: site%d has no idlst, its dense form is undefined" % i)
            dense = numpy.zeros(int(numpy.prod(lay.shape)))
            dense[lay.prjmap(idlst)] = values
            out["site%d" % i] = dense.reshape(tuple(int(n) for n in lay.shape))
        else:
            out["site%d" % i] = _read(node).astype(numpy.float64)
    return out
