"""Spin projection (SP-MPS): the oracle and the host-side operator builders pinned to
outputs of the reference itself (tests/golden/*SP_K*.npz, made by make_golden.py --spin)."""
import numpy
import pytest

from helpers import load, layout_of
from oracle.blocks import from_dict
from oracle import spin as ospin
from oracle.kernels import hdiag, RenormOracle
from qcmpodmrg_b200.hamiltonian import make_hamiltonian

TAGS = ["SP_K4", "SP_K5", "SPS_K4"]


def _quad(sw):
    return str(sw["quad"]) if "quad" in sw else "GaussLegendre"


def _ham(sw):
    return make_hamiltonian(int(sw["K"]), int(sw["N"]), int(sw["seed"]), None if sw["decay"] < 0 else sw["decay"])


def _blocks_by_q(rank, qsyms, blocks):
    """{(sector quantum numbers..., physical sector indices): block} -- order-free comparison."""
    out = {}
    for isyms, blk in blocks:
        key = tuple(tuple(numpy.rint(2 * qsyms[i][isyms[i]]).astype(int)) for i in range(rank))
        out[key + (tuple(int(x) for x in isyms[2:]),)] = blk
    return out


def _oracle_blocks(qt):
    return _blocks_by_q(qt.rank, qt.qsyms, [(isyms, qt.value[off:off + int(numpy.prod(d))].reshape(d))
                                            for idx, isyms, off, d in qt.blocks()])


def _layout_blocks(lay, vals):
    items = []
    for idx in lay.idx_allowed:
        isyms = numpy.unravel_index(idx, tuple(lay.nsyms))
        d = lay.block_dims(idx)[0]
        o = int(lay.ioff[idx])
        items.append((isyms, vals[o:o + int(numpy.prod(d))].reshape(d)))
    return _blocks_by_q(lay.rank, lay.qsyms, items)


@pytest.mark.parametrize("tag", TAGS)
def test_quadrature_matches_reference(tag):
    from qcmpodmrg_b200 import spin
    sw = load("sweep_%s.npz" % tag)
    r = load("kernels_%s.npz" % tag)["records"][0]
    for fn in (ospin.s2quad, spin.s2quad):
        pts, wts = fn(int(sw["npts"]), quad=_quad(sw))
        assert numpy.abs(pts - r["qpts"]).max() <= 1e-15
        assert numpy.abs(wts - r["qwts"]).max() <= 1e-15
    # Simpson and S > 0 agree between the two restatements
    for args in [(5, 0.0, 0.0, "Simpson"), (6, 1.0, 0.0, "GaussLegendre"), (4, 0.5, 0.5, "GaussLegendre")]:
        a, b = ospin.s2quad(*args), spin.s2quad(*args)
        assert numpy.abs(a[0] - b[0]).max() <= 1e-15 and numpy.abs(a[1] - b[1]).max() <= 1e-14


def test_smalld_known_values():
    from qcmpodmrg_b200.spin import smalld
    b = 0.7
    assert abs(smalld(0.5, 0.5, 0.5, b) - numpy.cos(b / 2)) < 1e-15
    assert abs(smalld(1, 1, 0, b) + numpy.sin(b) / numpy.sqrt(2)) < 1e-15
    assert abs(smalld(1, 0, 0, b) - numpy.cos(b)) < 1e-15
    assert abs(smalld(2, 0, 0, b) - 0.5 * (3 * numpy.cos(b) ** 2 - 1)) < 1e-14
    assert ospin.smalld(1, 0.5, 0, b) == 0.0


@pytest.mark.parametrize("tag", TAGS)
def test_sp_operators_match_reference(tag):
    """H_p R(theta_g) and R(theta_g), oracle and product builders, block by block."""
    from qcmpodmrg_b200 import spin
    sw = load("sweep_%s.npz" % tag)
    ham = _ham(sw)
    npts = int(sw["npts"])
    qpts, _ = spin.s2quad(npts, quad=_quad(sw))
    for r in load("kernels_%s.npz" % tag)["records"]:
        isite = int(r["key"][2])
        ops = ospin.sp_opers(ham.sbas, npts)
        assert [p for p, g in ops] == [int(x) for x in r["opers"]]
        assert numpy.array_equal([g for p, g in ops], r["opers_ipt"])
        for x, (p, g) in enumerate(ops):
            ref = _oracle_blocks(from_dict(r["mpo_i"][x]))
            a = _oracle_blocks(ospin.sp_site_operator(p, qpts[g], ham.sbas, isite, ham.int1e, ham.int2e))
            lay, vals = spin.sp_site_operator(p, qpts[g], ham.sbas, isite, ham.int1e, ham.int2e)
            b = _layout_blocks(lay, vals)
            assert a.keys() == ref.keys() == b.keys()
            assert max(numpy.abs(a[k] - ref[k]).max() for k in ref) == 0.0
            assert max(numpy.abs(b[k] - ref[k]).max() for k in ref) == 0.0
        for g in range(npts):
            ref = _oracle_blocks(from_dict(r["pop"][g]))
            assert all(numpy.array_equal(ospin.rotation_op(qpts[g]).block(i), from_dict(r["pop"][g]).block(i))
                       for i in from_dict(r["pop"][g]).idx_allowed)
            pset = spin.rotation_set(qpts, "cpu")
            b = _layout_blocks(pset.layouts[g], pset.op_values(g).numpy())
            assert b.keys() == ref.keys() and all(numpy.array_equal(b[k], ref[k]) for k in ref)


@pytest.mark.parametrize("tag", TAGS)
def test_sp_oracle_kernels_match_reference(tag):
    for r in load("kernels_%s.npz" % tag)["records"]:
        qtmp = from_dict(r["qtmp"])
        L, R = [from_dict(d) for d in r["envL"]], [from_dict(d) for d in r["envR"]]
        Wi, Wj = [from_dict(d) for d in r["mpo_i"]], [from_dict(d) for d in r["mpo_j"]]
        PL, PR = [from_dict(d) for d in r["penvL"]], [from_dict(d) for d in r["penvR"]]
        P = [from_dict(d) for d in r["pop"]]
        opers = [int(x) for x in r["opers"]]
        hp, qw = numpy.atleast_1d(r["hpwts"]), numpy.atleast_1d(r["qwts"])
        isite = int(r["key"][2])
        y = ospin.sigma_sp(qtmp, r["qkey"], L, R, Wi, Wj, opers, hp, isite)(r["hvec_x"])
        assert numpy.abs(y - r["hvec_y"]).max() <= 1e-12 * max(1.0, numpy.abs(r["hvec_y"]).max())
        s = ospin.svec(qtmp, r["qkey"], PL, PR, P, qw, isite)(r["svec_x"])
        assert numpy.abs(s - r["svec_y"]).max() <= 1e-13
        dims = tuple(int(x) for x in r["dims"])
        assert numpy.abs(hdiag(r["prjmap"], dims, L, R, Wi, Wj, hp) - r["hdiag"]).max() <= 1e-12
        assert numpy.abs(ospin.sdiag(r["prjmap"], dims, PL, PR, P, qw) - r["sdiag"]).max() <= 1e-13
        site = from_dict(r["renorm_site"]).reduce_to_n()
        if int(r["key"][1]) == 0:
            out = RenormOracle(opers, isite, "L")(site, L, Wi)
            pout = ospin.renorm_p(site, PL, P, isite, "L")
        else:
            out = RenormOracle(opers, isite + 1, "R")(site, R, Wj)
            pout = ospin.renorm_p(site, PR, P, isite + 1, "R")
        for a, b in list(zip(out, r["renorm_out"])) + list(zip(pout, r["renorm_pout"])):
            assert a.size_allowed == len(b["value"])
            assert numpy.abs(a.value - b["value"]).max() <= 1e-12


def test_sp_reduce_map_is_reference_reduction():
    """The product's scatter map reproduces reduceQsymsToN / projectionNMs."""
    from qcmpodmrg_b200.spin import reduce_layout, reduce_map
    r = load("kernels_SP_K5.npz")["records"][0]
    q = from_dict(r["qtmp"])
    q.value = numpy.random.default_rng(3).standard_normal(q.size_allowed)
    ref = q.reduce_to_n()
    lay = layout_of(r["qtmp"])
    lay_n = reduce_layout(lay)
    m = reduce_map(lay, lay_n)
    got = numpy.zeros(lay_n.size)
    got[m] = q.value
    assert lay_n.size == ref.size_allowed and numpy.array_equal(got, ref.value)
    assert numpy.array_equal(ref.projection_nms(q.qsyms).value, got[m])


def test_oracle_gdavidson_solves_generalised_problem():
    import scipy.linalg
    rng = numpy.random.default_rng(0)
    n = 80
    h = rng.uniform(-1, 1, (n, n))
    h = numpy.diag(numpy.arange(n) * 1.0) + h + h.T
    s = rng.uniform(0, 1, (n, n))
    s = numpy.diag(rng.uniform(0.8, 1.0, n)) + 0.05 * (s + s.T)
    e, v, nm = ospin.gdavidson(lambda x: h @ x, lambda x: s @ x, numpy.diag(h).copy(), 1, crit_e=1e-12,
                               crit_vec=1e-9, maxcycle=60)
    assert abs(e[0] - scipy.linalg.eigh(h, s, eigvals_only=True)[0]) < 1e-10
    assert abs(v[0] @ s @ v[0] - 1.0) < 1e-12


def test_sp_oracle_sweep_matches_reference():
    """K=4, 3 quadrature points, D=16 (no truncation), first R+L sweep: every dot energy,
    the averaged energy, weight and matvec count."""
    sw = load("sweep_SP_K4.npz")
    out = ospin.SPOracleDMRG(_ham(sw), int(sw["npts"])).run(sw["init_mps"], int(sw["D"]), 1)
    n = len(out["esweeps"])
    assert n == 2 * (int(sw["K"]) - 1)
    assert numpy.abs(out["esweeps"] - sw["esweeps"][:n]).max() <= 1e-8
    assert abs(out["eav"][0] - sw["eav"][0]) <= 1e-8 and abs(out["dwt"][0] - sw["dwt"][0]) <= 1e-10
    assert out["nmvp"][0] == sw["nmvp"][0]


@pytest.mark.parametrize("sval,npts", [(0.0, 3), (1.0, 4), (2.0, 6), (0.5, 4), (1.5, 5)])
def test_quadrature_projects_onto_total_spin(sval, npts):
    """sum_g w_g d^S'_{MM}(theta_g) = delta(S, S') for every S' the Gauss-Legendre rule
    integrates exactly (the projector's defining property, mpo_dmrg_util.py:35-89)."""
    from qcmpodmrg_b200.spin import s2quad, smalld
    m = sval - int(sval)                       # Sz = 0 or 1/2
    pts, wts = s2quad(npts, sval, m)
    for sp in numpy.arange(m, npts - 0.5, 1.0):
        got = sum(w * smalld(sp, m, m, t) for t, w in zip(pts, wts))
        assert abs(got - (1.0 if abs(sp - sval) < 1e-9 else 0.0)) <= 1e-12


def test_smalld_is_orthogonal():
    """d^j(beta) is a real orthogonal matrix in (m', m) for integer and half-integer j."""
    from qcmpodmrg_b200.spin import smalld
    for j in (0.5, 1.0, 1.5, 2.0, 3.0):
        ms = numpy.arange(-j, j + 0.5, 1.0)
        d = numpy.array([[smalld(j, a, b, 0.83) for b in ms] for a in ms])
        assert numpy.abs(d @ d.T - numpy.identity(len(ms))).max() <= 1e-13
