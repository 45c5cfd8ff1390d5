"""Seeded synthetic left-canonical MPS with (N, Sz) sectors of a realistic shape.

Used where no converged state of the requested bond dimension exists (the
D=500 and D=1000 benchmark workloads).  Bond i (after spatial orbital i) keeps
up to D states distributed over (N_L, Sz_L) sectors with Gaussian weights
around the mean filling N*(i+1)/K and Sz = 0, capped by what the left block can
hold and what the right block can complete; every site tensor has orthonormal
columns inside each symmetry sector (left-canonical), so the Qt sweep starts
from a valid state of the target symmetry.
"""
import numpy

QPHYS = numpy.array([[0., 0.], [1., -0.5], [1., 0.5], [2., 0.]])


def random_mps(K, N, D, seed=0, width=0.9, szwidth=0.6):
    rng = numpy.random.default_rng(seed)
    qnum = [numpy.zeros((1, 2))]
    sites = []
    for i in range(K):
        ql = qnum[-1]
        cand = (ql[:, None, :] + QPHYS[None, :, :]).reshape(-1, 2)        # (l, n) pairs
        keys, inv = numpy.unique(numpy.rint(2 * cand).astype(numpy.int64), axis=0, return_inverse=True)
        inv = inv.ravel()
        avail = numpy.bincount(inv, minlength=len(keys))
        rest = K - i - 1
        if i == K - 1:
            target = {(2 * N, 0): 1}
        else:
            nbar = N * (i + 1) / float(K)
            w = numpy.zeros(len(keys))
            for s, (n2, s2) in enumerate(keys):
                n, sz = n2 / 2.0, s2 / 2.0
                nr = N - n
                if nr < 0 or nr > 2 * rest or abs(sz) > min(n, 2 * (i + 1) - n) / 2.0 + 1e-9 \
                        or abs(sz) > min(nr, 2 * rest - nr) / 2.0 + 1e-9:
                    continue
                w[s] = numpy.exp(-0.5 * ((n - nbar) / width) ** 2 - 0.5 * (sz / szwidth) ** 2)
            if w.sum() == 0:
                raise ValueError("no admissible sector")
            w[w < 1e-3 * w.max()] = 0.0
            cnt = numpy.minimum(avail, numpy.floor(D * w / w.sum() + 0.5).astype(numpy.int64))
            while cnt.sum() > D:
                j = numpy.argmax(cnt)
                cnt[j] -= 1
            # fill up to D where room is left
            order = numpy.argsort(-w)
            k = 0
            while cnt.sum() < D and k < 100000:
                j = order[k % len(order)]
                if w[j] > 0 and cnt[j] < avail[j]:
                    cnt[j] += 1
                k += 1
                if k > 10 * len(order) and all(cnt[o] >= avail[o] or w[o] == 0 for o in order):
                    break
            target = {tuple(keys[s]): int(cnt[s]) for s in range(len(keys)) if cnt[s] > 0}
        ldim = len(ql)
        cols, qr = [], []
        for key in sorted(target):
            rows = numpy.flatnonzero((numpy.rint(2 * cand).astype(numpy.int64) == numpy.array(key)).all(axis=1))
            m = target[key]
            if len(rows) == 0:
                continue
            m = min(m, len(rows))
            q, _ = numpy.linalg.qr(rng.standard_normal((len(rows), m)))
            col = numpy.zeros((ldim * 4, m))
            col[rows, :] = q
            cols.append(col)
            qr += [numpy.array(key) / 2.0] * m
        mat = numpy.hstack(cols)
        sites.append(mat.reshape(ldim, 4, -1))
        qnum.append(numpy.array(qr))
    out = {"site%d" % i: s for i, s in enumerate(sites)}
    out.update({"qnum%d" % i: q for i, q in enumerate(qnum)})
    return out


def product_mps(ham):
    """The occupation-number (Hartree-Fock) product state as a bond-dimension-1 L-MPS
    (the reference's mps0occun, source/mpo_dmrg_util.py:118-156)."""
    K = ham.nsite
    occ = ham.occun
    qnum = [numpy.zeros((1, 2))]
    sites = {}
    n, sz = 0.0, 0.0
    for i in range(K):
        na, nb = occ[2 * i], occ[2 * i + 1]
        t = numpy.zeros((1, 4, 1))
        if na < 0.5 and nb < 0.5:
            t[0, 0, 0] = 1.0
        elif na < 0.5:
            t[0, 1, 0] = 1.0
            n, sz = n + 1, sz - 0.5
        elif nb < 0.5:
            t[0, 2, 0] = 1.0
            n, sz = n + 1, sz + 0.5
        else:
            t[0, 3, 0] = 1.0
            n += 2
        sites["site%d" % i] = t
        qnum.append(numpy.array([[n, sz]]))
    sites.update({"qnum%d" % i: q for i, q in enumerate(qnum)})
    return sites
