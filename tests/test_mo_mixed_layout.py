"""CPU restatement of the operand layouts of the split-BF16 MO transforms (rerdmft_b200/csrc/mo_mixed.cu), in
exact FP64 arithmetic: the two flat real GEMMs with the kernels' index maps reproduce the oracle's
buildRiNonRelSpinMoEri (src/NON_REL/NonRelSpinRiMoEri.cpp:13-43) and buildRiMoEri (src/UKB/RiMoEri.cpp:20-86)
element for element, for non-symmetric B^P as well.  The BF16 rounding itself is checked on the GPU
(tests/test_gpu_mo_mixed.py)."""
import numpy as np
import pytest

from oracle import ri_oracle as o


def _nonrel_two_step(B, C):
    naux, n = B.shape[0], C.shape[0]
    Bt = B.reshape(naux, n, n).transpose(0, 2, 1)   # resident split copy: Bt[P][a][q] = B[P][q][a]
    Ct = C.T                                         # B operand rows j: Ct[j][q] = C[q][j]
    Y = np.einsum("Paq,jq->Paj", Bt, Ct)             # step 1 rows (P, a), columns j
    Yt = Y.transpose(0, 2, 1)                        # EPI 0 store: Yt[P][j][a]
    O = np.einsum("Pja,ia->Pji", Yt, Ct)             # step 2 rows (P, j), columns i
    return O.reshape(naux, n * n)                    # EPI 1 store: B_mo[P][j][i]


def _ukb_two_step(nl, ns, B_LL, B_SS, c):
    naux, nt = B_LL.shape[0], c.shape[1]
    nu = 2 * nl + 2 * ns
    off, fs = [0, nl, 2 * nl, 2 * nl + ns], [nl, nl, ns, ns]
    cc = np.zeros((2 * nt, 2 * nu))                  # cc_split_kernel
    cc[0::2, :nu], cc[0::2, nu:] = c.real.T, c.imag.T
    cc[1::2, :nu], cc[1::2, nu:] = -c.imag.T, c.real.T
    Yt = np.zeros((naux, nt, 2 * nu))
    for f in range(4):
        if fs[f] == 0:
            continue
        Bf = (B_LL if f < 2 else B_SS).reshape(naux, fs[f], fs[f])
        blk = c[off[f]:off[f] + fs[f]]
        ct2 = np.concatenate([blk.real.T, blk.imag.T])               # ct2_split_kernel: 2 nt rows
        Y = np.einsum("Paq,jq->Paj", Bf.transpose(0, 2, 1), ct2)     # step 1 rows (P, a), columns j'
        for col in range(2 * nt):                                    # EPI 0 with cmod = nt, chi = nu, koff = off_f
            k0 = (col // nt) * nu + off[f]
            Yt[:, col % nt, k0:k0 + fs[f]] = Y[:, :, col]
    O = np.einsum("Pqk,ik->Pqi", Yt, cc)                            # step 2 rows (P, q), columns (p, Re / Im)
    O[:, :, 1::2] *= -1.0                                            # EPI 1 conj_odd
    return (O[:, :, 0::2] + 1j * O[:, :, 1::2]).reshape(naux, nt * nt)


@pytest.mark.parametrize("n,naux", [(1, 2), (7, 5), (16, 9)])
def test_nonrel_layout_reproduces_oracle(n, naux):
    rng = np.random.default_rng(n)
    B = rng.standard_normal((naux, n * n))          # not symmetric
    C = rng.standard_normal((n, n))
    assert np.abs(_nonrel_two_step(B, C) - o.nonrel_mo_build(B, C)).max() <= 1e-12


@pytest.mark.parametrize("nl,ns,naux,nt", [(2, 3, 4, 3), (5, 7, 6, 9), (4, 0, 3, 5)])
def test_ukb_layout_reproduces_oracle(nl, ns, naux, nt):
    rng = np.random.default_rng(nl + ns)
    B_LL = rng.standard_normal((naux, nl * nl))     # not symmetric
    B_SS = rng.standard_normal((naux, ns * ns))
    nu = 2 * nl + 2 * ns
    c = rng.standard_normal((nu, nt)) + 1j * rng.standard_normal((nu, nt))
    got = _ukb_two_step(nl, ns, B_LL, B_SS, c)
    ref = o.ri_mo_build(nl, ns, B_LL, B_SS, c)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_column_tile_cost_model():
    """The column-tile choice of mo_mixed.cu's pick_bn: cost ntn * (BN + 64) over the instantiated widths,
    the order measured at n = 400 (208 < 144 < 256 < 112 < 128)."""
    def pick(n):
        best, cost = 256, -(-n // 256) * 320
        for c in (32, 64, 112, 128, 144, 208, 256):
            k = -(-n // c) * (c + 64)
            if k < cost:
                best, cost = c, k
        return best
    assert pick(400) == 208 and pick(800) == 208 and pick(24) == 32 and pick(130) == 144
    costs = {c: -(-400 // c) * (c + 64) for c in (208, 144, 256, 112, 128)}
    assert sorted(costs, key=costs.get) == [208, 144, 256, 112, 128]


def _bf16(x):
    """Round-to-nearest-even to BF16 (through FP32), as __float2bfloat16_rn / __double2bfloat16 do for these
    magnitudes."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _split_mm(A, B):
    """Three BF16 products hi hi + hi lo + lo hi with FP32 accumulation."""
    ah, bh = _bf16(A), _bf16(B)
    al, bl = _bf16(A - ah), _bf16(B - bh)
    f = lambda a, b: (a.astype(np.float32) @ b.astype(np.float32)).astype(np.float64)  # noqa: E731
    return f(ah, bh) + f(ah, bl) + f(al, bh)


@pytest.mark.parametrize("n,naux", [(24, 6), (64, 3)])
def test_split_bf16_error_model(n, naux):
    """The rounding model behind the GPU tolerance (3e-5 of max|B_mo|): step 1 in split BF16, its FP32 result
    re-split, step 2 in split BF16.  The emulation stays well inside the bound (about 1e-5)."""
    from rerdmft_b200 import synth

    rng = np.random.default_rng(n)
    B = synth.ri_tensor(n, naux, n, box=6.0)
    C = synth.random_orthogonal(n, rng)
    ref = o.nonrel_mo_build(B, C).reshape(naux, n, n)
    for P in range(naux):
        BP = B[P].reshape(n, n)
        Y = _split_mm(BP.T, C).astype(np.float32).astype(np.float64)   # step 1, FP32 accumulator
        got = _split_mm(Y.T, C)                                         # step 2: rows j, columns i, stored [j][i]
        assert np.abs(got - ref[P]).max() <= 3e-5 * np.abs(ref).max()
