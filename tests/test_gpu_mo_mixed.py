"""The split-BF16 (RR_PREC_MIXED) MO three-index transforms on the tensor cores: B_mo^P = C^T B^P C against
the numpy restatement of buildRiNonRelSpinMoEri (src/NON_REL/NonRelSpinRiMoEri.cpp:13-43) and the FP64 device
build, the in-place rebuild of an existing MO tensor, and the complex buildRiMoEri (src/UKB/RiMoEri.cpp:20-86)
against its restatement and the FP64 device build.

Tolerance: three BF16 products with FP32 accumulation per product and the intermediate C^T B^P re-split
to BF16 pairs give a relative error of about 1e-5 of max|B_mo| (a numpy emulation of the same rounding
gives 7e-6 to 9e-6 on these shapes); the tests hold it to MIXED_REL = 3e-5 of max|B_mo|."""
import numpy as np
import pytest

from oracle import ri_oracle as o
from rerdmft_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from rerdmft_b200 import _lib as L  # noqa: E402
from rerdmft_b200 import mo, ri  # noqa: E402

MIXED_REL = 3e-5
TOL = 1e-10


@pytest.mark.parametrize("n,naux", [(1, 3), (24, 129), (33, 200), (64, 77), (130, 333), (257, 64)])
def test_mixed_mo_build_vs_oracle(n, naux):
    rng = np.random.default_rng(1000 + n)
    B = synth.ri_tensor(n, naux, n, box=6.0)
    C = synth.random_orthogonal(n, rng)
    src = ri.RiNonRelEriSource(n, B, np.eye(n), np.eye(n))
    m = mo.buildRiNonRelSpinMoEri(src, n, C, precision=L.RR_PREC_MIXED)
    ref = o.nonrel_mo_build(B, C)
    err = float(np.abs(m.b() - ref).max())
    scale = max(float(np.abs(ref).max()), 1e-300)
    print(f"n={n} naux={naux}: max|B_mo(mixed) - B_mo(FP64 oracle)| = {err:.3e} ({err / scale:.2e} of max)")
    assert err <= MIXED_REL * scale
    # a non-symmetric B^P and a non-orthogonal C: the product is C^T B^P C element for element
    Bn = rng.standard_normal((naux, n * n))
    Cn = rng.standard_normal((n, n))
    srcn = ri.RiNonRelEriSource(n, Bn, np.eye(n), np.eye(n))
    refn = np.einsum("ai,pab,bj->pij", Cn, Bn.reshape(naux, n, n), Cn, optimize=True).reshape(naux, n * n)
    gotn = mo.buildRiNonRelSpinMoEri(srcn, n, Cn, precision=L.RR_PREC_MIXED).b()
    bound = np.einsum("ai,pab,bj->pij", np.abs(Cn), np.abs(Bn.reshape(naux, n, n)), np.abs(Cn),
                      optimize=True).reshape(naux, n * n)
    assert np.all(np.abs(gotn - refn) <= MIXED_REL * bound + 1e-300)


def test_mixed_mo_build_headline_shape():
    """n = 400, naux = 1600: the shape of the nonrelativistic headline build (BN = 208 column tiles,
    5000 row tiles per step), against the FP64 device build (itself pinned to the reference)."""
    n, naux = 400, 1600
    rng = np.random.default_rng(7)
    B = synth.ri_tensor(n, naux, n, box=20.0)
    C = synth.random_orthogonal(n, rng)
    dB = torch.from_numpy(B).cuda()
    st = ri.RiStore(dB, nl=n)
    dC = torch.from_numpy(C).cuda()
    f64 = mo.buildRiNonRelSpinMoEri(st, n, dC)
    mx = mo.buildRiNonRelSpinMoEri(st, n, dC, precision=L.RR_PREC_MIXED)
    a, b = f64.b(), mx.b()
    err = float(np.abs(a - b).max())
    scale = float(np.abs(a).max())
    print(f"n=400 naux=1600: max|B_mo(mixed) - B_mo(FP64)| = {err:.3e} ({err / scale:.2e} of max)")
    assert err <= MIXED_REL * scale
    # spot check of the FP64 build against the restatement on a few aux rows
    rows = [0, 777, naux - 1]
    ref = o.nonrel_mo_build(B[rows], C)
    assert np.abs(a[rows] - ref).max() <= TOL
    st.close()


@pytest.mark.parametrize("precision", [L.RR_PREC_FP64, L.RR_PREC_MIXED])
def test_rebuild_into_existing_tensor(precision):
    n, naux = 48, 150
    rng = np.random.default_rng(3)
    B = synth.ri_tensor(n, naux, n, box=6.0)
    src = ri.RiNonRelEriSource(n, B, np.eye(n), np.eye(n))
    C1, C2 = synth.random_orthogonal(n, rng), synth.random_orthogonal(n, rng)
    m = mo.buildRiNonRelSpinMoEri(src, n, C1, precision=precision)
    fresh = mo.buildRiNonRelSpinMoEri(src, n, C2, precision=precision).b()
    again = mo.buildRiNonRelSpinMoEri(src, n, C2, precision=precision, into=m)
    assert again is m
    assert np.array_equal(m.b(), fresh)  # same kernels, same order: bit-identical
    # device-pointer form, twice in a row
    dC = torch.from_numpy(C1).cuda()
    mo.buildRiNonRelSpinMoEri(src, n, dC, precision=precision, into=m)
    mo.buildRiNonRelSpinMoEri(src, n, dC, precision=precision, into=m)
    ref = o.nonrel_mo_build(B, C1)
    tol = TOL if precision == L.RR_PREC_FP64 else MIXED_REL * np.abs(ref).max()
    assert np.abs(m.b() - ref).max() <= tol


def test_rebuild_into_rejects_other_shapes():
    n = 12
    B = synth.ri_tensor(n, 40, n, box=6.0)
    src = ri.RiNonRelEriSource(n, B, np.eye(n), np.eye(n))
    other = mo.buildRiNonRelSpinMoEri(ri.RiNonRelEriSource(n, B[:30], np.eye(n), np.eye(n)), n, np.eye(n))
    with pytest.raises(L.RrError, match="rr_mo_build_nonrel_into"):
        mo.buildRiNonRelSpinMoEri(src, n, np.eye(n), into=other)


@pytest.mark.parametrize("nl,ns,naux,nt", [(3, 5, 7, 4), (12, 20, 50, 17), (33, 70, 40, 64), (64, 130, 30, 100)])
def test_mixed_ukb_build_vs_oracle(nl, ns, naux, nt):
    rng = np.random.default_rng(nl + ns)
    B_LL = synth.ri_tensor(nl, naux, nl, box=6.0)
    B_SS = synth.ri_tensor(ns, naux, ns, box=6.0)
    c = synth.random_unitary(2 * nl + 2 * ns, rng)[:, :nt]
    src = ri.RiDirectEriSource(nl, ns, B_LL, B_SS)
    got = mo.buildRiMoEri(src, c, precision=L.RR_PREC_MIXED).b()
    ref = o.ri_mo_build(nl, ns, B_LL, B_SS, c)
    err = float(np.abs(got - ref).max())
    scale = float(np.abs(ref).max())
    print(f"nl={nl} ns={ns} naux={naux} nt={nt}: max|B(mixed) - B(FP64 oracle)| = {err:.3e} ({err / scale:.2e} of max)")
    assert err <= MIXED_REL * scale
    # non-symmetric B^P blocks: the stored tensor is c^dagger B^P c element for element
    Bn_LL, Bn_SS = rng.standard_normal((naux, nl * nl)), rng.standard_normal((naux, ns * ns))
    srcn = ri.RiDirectEriSource(nl, ns, Bn_LL, Bn_SS)
    gotn = mo.buildRiMoEri(srcn, c, precision=L.RR_PREC_MIXED).b()
    refn = o.ri_mo_build(nl, ns, Bn_LL, Bn_SS, c)
    bound = o.ri_mo_build(nl, ns, np.abs(Bn_LL), np.abs(Bn_SS), np.abs(c)).real  # sum of |terms| per element
    assert np.all(np.abs(gotn - refn) <= MIXED_REL * bound)


def test_mixed_ukb_build_large():
    """nl = 100, ns = 300, naux = 200, 200 spinors: 2 nt = 400 columns (BN = 208), K = 2 n_ukb = 1600, against
    the FP64 device build."""
    nl, ns, naux, nt = 100, 300, 200, 200
    rng = np.random.default_rng(11)
    B_LL = synth.ri_tensor(nl, naux, 1, box=12.0)
    B_SS = synth.ri_tensor(ns, naux, 2, box=12.0)
    c = synth.random_unitary(2 * nl + 2 * ns, rng)[:, :nt]
    src = ri.RiDirectEriSource(nl, ns, B_LL, B_SS)
    a = mo.buildRiMoEri(src, c).b()
    b = mo.buildRiMoEri(src, c, precision=L.RR_PREC_MIXED).b()
    err = float(np.abs(a - b).max())
    scale = float(np.abs(a).max())
    print(f"nl=100 ns=300 naux=200 nt=200: max|B(mixed) - B(FP64)| = {err:.3e} ({err / scale:.2e} of max)")
    assert err <= MIXED_REL * scale
