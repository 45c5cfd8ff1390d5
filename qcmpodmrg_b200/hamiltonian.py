"""Seeded synthetic ab-initio Hamiltonians in the reference's spin-orbital format.

Spatial integrals (K orbitals), drawn from ``numpy.random.default_rng(seed)``
in this fixed order:
  1. h1e diagonal  ~ U(-2, -0.5)            (K draws)
  2. h1e upper off-diagonal ~ N(0, 0.1)     (K*K draws, upper triangle used)
  3. for k in range(3K): B_k upper ~ N(0, 0.05) (K*K draws each, upper used)
h1e and every B_k are symmetric; the ERI (pq|rs) = sum_k B_k[p,q] B_k[r,s] is
8-fold symmetric and positive semidefinite.  With a locality decay length
``decay`` every h1e[p,q] and B_k[p,q] is multiplied by exp(-|p-q|/decay).

The spin-orbital conversion follows the reference's integral dump
(source/itools/ipyscf_real.py:202-241): spin orbital 2i is alpha and 2i+1 is
beta of spatial orbital i; one-electron mixed-spin blocks are zero; the ERI in
chemist order has its mixed-spin pairs zeroed, is transposed to physicist order
<pq|rs> = (pr|qs) and antisymmetrised as V[pqrs] = -1/2 (<pq|rs> - <pq|sr>).
The initial occupation puts N/2 electrons of each spin in the first spatial
orbitals (ipyscf_real.py:170-174 with no reordering).
"""
import numpy


class SpinOrbitalHamiltonian(object):
    """Integrals and metadata of one synthetic molecule (the reference's mole.h5 content)."""

    def __init__(self, int1e, int2e, nelec, occun, enuc=0.0):
        self.int1e = int1e          # (2K, 2K)
        self.int2e = int2e          # (2K, 2K, 2K, 2K)
        self.nelec = nelec
        self.sbas = int1e.shape[0]
        self.nsite = self.sbas // 2
        self.occun = occun
        self.enuc = enuc
        self.ecor = 0.0
        self.escf = 0.0


def spatial_integrals(K, seed, decay=None):
    rng = numpy.random.default_rng(seed)
    h = numpy.zeros((K, K))
    h[numpy.diag_indices(K)] = rng.uniform(-2.0, -0.5, size=K)
    off = rng.normal(0.0, 0.1, size=(K, K))
    iu = numpy.triu_indices(K, 1)
    h[iu] = off[iu]
    h[(iu[1], iu[0])] = off[iu]
    B = numpy.zeros((3 * K, K, K))
    iu0 = numpy.triu_indices(K, 0)
    for k in range(3 * K):
        m = rng.normal(0.0, 0.05, size=(K, K))
        B[k][iu0] = m[iu0]
        B[k][(iu0[1], iu0[0])] = m[iu0]
    if decay is not None:
        idx = numpy.arange(K)
        fac = numpy.exp(-numpy.abs(idx[:, None] - idx[None, :]) / float(decay))
        h = h * fac
        B = B * fac[None, :, :]
    eri = numpy.einsum("kpq,krs->pqrs", B, B)
    return h, eri


def to_spin_orbital(h, eri):
    K = h.shape[0]
    n = 2 * K
    hmo = numpy.zeros((n, n))
    hmo[0::2, 0::2] = h
    hmo[1::2, 1::2] = h
    e = numpy.zeros((n, n, n, n))
    for s1 in range(2):
        for s2 in range(2):
            e[s1::2, s1::2, s2::2, s2::2] = eri
    e = e.transpose(0, 2, 1, 3)
    v = -0.5 * (e - e.transpose(0, 1, 3, 2))
    return hmo, numpy.ascontiguousarray(v)


def make_hamiltonian(K, N, seed, decay=None):
    """Build the synthetic Hamiltonian of K spatial orbitals and N electrons; the start
    occupation fills spin orbitals 0..N-1 (alpha, beta alternating: Sz = 0 for even N,
    +1/2 for odd N)."""
    if not 0 <= N <= 2 * K:
        raise ValueError("need 0 <= N <= 2K")
    h, eri = spatial_integrals(K, seed, decay)
    int1e, int2e = to_spin_orbital(h, eri)
    occun = numpy.zeros(2 * K)
    occun[: N] = 1.0
    return SpinOrbitalHamiltonian(int1e, int2e, N, occun)


def fci_energy(ham):
    """Exact ground energy in the determinant space of N electrons with N//2 alpha ones
    (Sz = 0, or -1/2 for odd N; small K only).

    Independent check used by the tests: DMRG with an unrestricted bond
    dimension must reproduce it.
    """
    h, dets = fci_hamiltonian(ham)
    return numpy.linalg.eigvalsh(h)[0]


def fci_hamiltonian(ham):
    """H in the basis of determinants with N//2 alpha electrons (Sz = 0, or -1/2 for odd
    N; sorted spin-orbital tuples, 2i = alpha, 2i+1 = beta), symmetrised, and the
    determinants."""
    from itertools import combinations
    n = ham.sbas
    N = ham.nelec
    na = N // 2
    alpha = [2 * i for i in range(n // 2)]
    beta = [2 * i + 1 for i in range(n // 2)]
    dets = []
    for oa in combinations(alpha, na):
        for ob in combinations(beta, N - na):
            dets.append(tuple(sorted(oa + ob)))
    index = {d: i for i, d in enumerate(dets)}
    # H = sum_pq h_pq a+_p a_q + sum_{pqrs} V'_{pqrs} a+_p a+_q a_r a_s with
    # <pq||rs> = -2 V[pqrs]:  H2 = 1/4 sum <pq||rs> a+p a+q a_s a_r
    h = ham.int1e
    g = -2.0 * ham.int2e          # <pq||rs>
    dim = len(dets)
    H = numpy.zeros((dim, dim))

    def apply(det, ops):
        # ops: list of (orb, dagger) applied right-to-left
        occ = list(det)
        sign = 1
        for orb, dag in reversed(ops):
            if dag:
                if orb in occ:
                    return None, 0
                pos = sum(1 for o in occ if o < orb)
                sign *= (-1) ** pos
                occ.append(orb)
                occ.sort()
            else:
                if orb not in occ:
                    return None, 0
                pos = occ.index(orb)
                sign *= (-1) ** pos
                occ.remove(orb)
        return tuple(occ), sign

    for j, dj in enumerate(dets):
        for p in range(n):
            for q in range(n):
                if h[p, q] == 0.0:
                    continue
                d, s = apply(dj, [(p, True), (q, False)])
                if d is not None and d in index:
                    H[index[d], j] += s * h[p, q]
        occ = list(dj)
        for r in occ:
            for s_ in occ:
                if s_ <= r:
                    continue
                for p in range(n):
                    for q in range(p + 1, n):
                        val = g[p, q, r, s_]
                        if val == 0.0:
                            continue
                        d, sg = apply(dj, [(p, True), (q, True), (s_, False), (r, False)])
                        if d is not None and d in index:
                            H[index[d], j] += sg * val
    return 0.5 * (H + H.T), dets
