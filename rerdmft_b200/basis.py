"""Orbital and auxiliary Gaussian basis sets on the host: the inputs of the device integral engine
(``integrals.py``), as the reference lays them out.

* ``read_basis_set``          src/AO_basis/BasisSet.cpp:27-160 (Gaussian94 ``.gbs`` files; SP / L shells
                              split into an S and a P shell; Fortran ``D`` exponents; the shell scale
                              factor squared onto the exponents)
* ``build_molecular_basis``   src/AO_basis/MolecularBasis.cpp:8-27 (one entry per Cartesian component,
                              atoms in input order, shells in file order, components in
                              ``cartesian_components`` order)
* ``group_into_shells``       src/AO_basis/MolecularBasis.cpp:29-58
* ``normalize_cartesian_basis``  src/AO_ints/Integrals.cpp:140-187 (libcint's conventions: primitive
                              radial normalisation, then each Cartesian component scaled to unit
                              self-overlap, the overlap carrying libcint's s / p factor)
* ``build_auto_auxiliary_basis``  src/AO_basis/AuxiliaryBasis.cpp:116-190 (the AUTO / PAUTO recipe)
* ``build_spherical_transform``  src/Utils/SphericalTransform.cpp:60-165 (per l: the Laplacian's null space on
                              the monomials, Loewdin-orthonormalised in the normalised Cartesian overlap)
* ``ANGSTROM_TO_BOHR``        src/Input/Input.cpp:23

A basis is a list of :class:`BasisFunction` (the reference's struct of the same name); ``flatten``
turns one into the plain arrays the C ABI takes (``rr_basis`` in include/rr_ri.h).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

ANGSTROM_TO_BOHR = 1.0 / 0.52917721067

_SYMBOLS = ("H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
            "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
            "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr Rf "
            "Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()
_LETTERS = "SPDFGHI"


def atomic_number(symbol: str) -> int:
    """Nuclear charge of an element symbol, case-insensitive (src/Utils/Element.cpp:27-35)."""
    up = symbol.upper()
    for i, s in enumerate(_SYMBOLS):
        if s.upper() == up:
            return i + 1
    raise ValueError(f"unrecognized element symbol '{symbol}'")


@dataclass
class Shell:
    """A contracted shell as read from the file: coefficients as given (src/AO_basis/Shell.h:10-14)."""
    l: int
    exponents: list = field(default_factory=list)
    coefficients: list = field(default_factory=list)


@dataclass
class Atom:
    symbol: str
    x: float
    y: float
    z: float


@dataclass
class BasisFunction:
    """One contracted Cartesian function at a centre (src/AO_basis/MolecularBasis.h:13-22)."""
    element: str
    x: float
    y: float
    z: float
    l: int
    cartesian: tuple
    exponents: list
    coefficients: list


def cartesian_components(l: int) -> list:
    """(lx, ly, lz) with lx + ly + lz = l in libcint's order: x-major, then y (src/AO_basis/Shell.cpp:5-14)."""
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def _strip_comment(line: str) -> str:
    cut = min([i for i in (line.find("#"), line.find("!")) if i >= 0], default=len(line))
    return line[:cut].strip()


def _fortran_float(tok: str) -> float:
    return float(tok.replace("D", "e").replace("d", "e"))


def read_basis_set(path: str) -> dict:
    """{ELEMENT (upper case): [Shell, ...]} from a Gaussian94 basis file."""
    with open(path) as f:
        lines = [_strip_comment(x) for x in f]
    lines = [x for x in lines if x]
    sep = lambda s: set(s) == {"*"}  # noqa: E731
    out: dict = {}
    i = 0
    while i < len(lines):
        if sep(lines[i]):
            i += 1
            continue
        symbol = lines[i].split()[0].upper()
        if symbol in out:
            raise ValueError(f"duplicate basis definition for element '{symbol}'")
        i += 1
        shells = []
        while i < len(lines) and not sep(lines[i]):
            head = lines[i].split()
            if len(head) < 3:
                raise ValueError(f"malformed shell header '{lines[i]}'")
            kind, nprim, scale = head[0].upper(), int(head[1]), float(head[2])
            i += 1
            is_sp = kind in ("SP", "L")
            if not is_sp and (len(kind) != 1 or kind not in _LETTERS):
                raise ValueError(f"unsupported shell type '{kind}'")
            rows = [lines[i + k].split() for k in range(nprim)]
            i += nprim
            exps = [_fortran_float(r[0]) for r in rows]
            if scale != 1.0:
                exps = [e * scale * scale for e in exps]
            if is_sp:
                shells.append(Shell(0, list(exps), [_fortran_float(r[1]) for r in rows]))
                shells.append(Shell(1, list(exps), [_fortran_float(r[2]) for r in rows]))
            else:
                shells.append(Shell(_LETTERS.index(kind), exps, [_fortran_float(r[1]) for r in rows]))
        if not shells:
            raise ValueError(f"element '{symbol}' has no shells")
        out[symbol] = shells
        i += 1
    return out


def basis_set_from_arrays(shell_element, shell_l, shell_nprim, exponents, coefficients) -> dict:
    """{ELEMENT: [Shell, ...]} from flat per-shell arrays (element, l, primitive count) and the concatenated
    exponents and coefficients, the inverse of listing read_basis_set's shells in order."""
    out: dict = {}
    off = 0
    for el, l, npr in zip(shell_element, shell_l, shell_nprim):
        npr = int(npr)
        out.setdefault(str(el).upper(), []).append(
            Shell(int(l), [float(v) for v in exponents[off:off + npr]], [float(v) for v in coefficients[off:off + npr]]))
        off += npr
    return out


def build_molecular_basis(geometry: list, basis_set: dict) -> list:
    """Copies each atom's shells to its position, one BasisFunction per Cartesian component."""
    fns = []
    for atom in geometry:
        key = atom.symbol.upper()
        if key not in basis_set:
            raise ValueError(f"no basis functions for element '{atom.symbol}'")
        for sh in basis_set[key]:
            for c in cartesian_components(sh.l):
                fns.append(BasisFunction(atom.symbol, atom.x, atom.y, atom.z, sh.l, c, list(sh.exponents),
                                         list(sh.coefficients)))
    return fns


def group_into_shells(basis: list) -> list:
    """[(first, count)] runs of consecutive components sharing centre, l and exponents."""
    out, i = [], 0
    while i < len(basis):
        f0 = basis[i]
        cnt = len(cartesian_components(f0.l))
        if i + cnt > len(basis):
            raise ValueError("group_into_shells: basis list ends mid-shell")
        for m in basis[i + 1:i + cnt]:
            if (m.l, m.x, m.y, m.z) != (f0.l, f0.x, f0.y, f0.z) or m.exponents != f0.exponents:
                raise ValueError("group_into_shells: basis list is not laid out as consecutive shells")
        out.append((i, cnt))
        i += cnt
    return out


def libcint_common_factor(l: int) -> float:
    """libcint evaluates coefficient * f(l) * x^lx y^ly z^lz exp(-a r^2) with f = 1/sqrt(4 pi) for s,
    sqrt(3 / (4 pi)) for p and 1 above (the reference states this at src/Utils/AIMPAC.cpp:100-106)."""
    if l == 0:
        return 1.0 / math.sqrt(4.0 * math.pi)
    if l == 1:
        return math.sqrt(3.0 / (4.0 * math.pi))
    return 1.0


def radial_norm(l: int, a: float) -> float:
    """1 / sqrt(int_0^inf r^(2l+2) exp(-2 a r^2) dr) = sqrt(2 (2a)^(l+3/2) / Gamma(l+3/2)): the primitive
    normalisation normalize_cartesian_basis applies (libcint's CINTgto_norm)."""
    return math.sqrt(2.0 * (2.0 * a) ** (l + 1.5) / math.gamma(l + 1.5))


def _double_factorial_odd(k: int) -> float:
    """(2k - 1)!!, 1 for k = 0."""
    r = 1.0
    for j in range(1, 2 * k, 2):
        r *= j
    return r


def cartesian_self_overlap(l: int, comp: tuple, exponents, coefficients) -> float:
    """<phi|phi> in libcint's convention for phi = f(l) sum_p c_p x^lx y^ly z^lz exp(-a_p r^2) at one centre:
    f(l)^2 sum_pq c_p c_q prod_d (2 l_d - 1)!! / (2 s)^l_d sqrt(pi / s), s = a_p + a_q."""
    a = np.asarray(exponents, dtype=np.float64)
    c = np.asarray(coefficients, dtype=np.float64)
    s = a[:, None] + a[None, :]
    val = np.ones_like(s)
    for ld in comp:
        val = val * (_double_factorial_odd(ld) / (2.0 * s) ** ld * np.sqrt(math.pi / s))
    return float(libcint_common_factor(l) ** 2 * (c[:, None] * c[None, :] * val).sum())


def normalize_cartesian_basis(functions: list, tolerance: float = 1e-10) -> list:
    """In place, per consecutive group of len(cartesian_components(l)) functions (the first one's
    exponents and coefficients stand for the group): c_p <- c_p radial_norm(l, a_p), then each component
    k scaled by 1 / sqrt(S_kk).  Returns [(element, l, cartesian, S_kk, renormalized)]."""
    report = []
    i = 0
    while i < len(functions):
        f0 = functions[i]
        l = f0.l
        if l > 6:
            raise ValueError(f"angular momentum l={l} exceeds the supported maximum (l=6, i-type)")
        comps = cartesian_components(l)
        exps = list(f0.exponents)
        coefs = [c * radial_norm(l, a) for c, a in zip(f0.coefficients, exps)]
        for k, comp in enumerate(comps):
            s_kk = cartesian_self_overlap(l, comp, exps, coefs)
            scale = 1.0 / math.sqrt(s_kk)
            fn = functions[i + k]
            fn.exponents = list(exps)
            fn.coefficients = [c * scale for c in coefs]
            report.append((fn.element, l, fn.cartesian, s_kk, abs(s_kk - 1.0) > tolerance))
        i += len(comps)
    return report


def _lval(z: int) -> int:
    return 0 if z <= 2 else 1 if z <= 18 else 2 if z <= 54 else 3


def _cluster(cands: list, f_sam: float, lmax_abs: int) -> list:
    """The greedy clustering of the AUTO / PAUTO recipe (src/AO_basis/AuxiliaryBasis.cpp:73-127):
    largest remaining exponent, absorb every remaining candidate within ratio f_sam, geometric mean of
    the unique (exponent, am) pairs (in log space), am = min(max(am in cluster, running am), lmax_abs)."""
    remaining = [True] * len(cands)
    left = len(cands)
    am_current = 0
    groups = []
    while left > 0:
        idx, best = 0, -1.0
        for k, (e, _) in enumerate(cands):
            if remaining[k] and e > best:
                best, idx = e, k
        e_cur = cands[idx][0]
        trial = [idx]
        remaining[idx] = False
        left -= 1
        for k, (e, _) in enumerate(cands):
            if remaining[k] and e_cur / e < f_sam:
                trial.append(k)
                remaining[k] = False
                left -= 1
        unique = []
        for t in trial:
            e, am = cands[t]
            if not any(u_am == am and abs(u_e - e) < 1e-6 for u_e, u_am in unique):
                unique.append((e, am))
        e_sel = math.exp(sum(math.log(e) for e, _ in unique) / len(unique))
        am_sel = min(max(max(cands[t][1] for t in trial), am_current), lmax_abs)
        am_current = am_sel
        groups.append((e_sel, am_sel))
    return groups


def build_auto_auxiliary_basis(orbital_basis: list, kind: str = "PAUTO", f_sam: float = 1.5,
                               lmax_inc: int = 1) -> list:
    """Automatic RI auxiliary basis per centre (Yang, Rendell, Frisch, J. Chem. Phys. 127, 074102 (2007)).
    Candidates: PAUTO every ordered pair of the centre's shells and of their primitives
    (a_i + a_j, l_i + l_j); AUTO each primitive doubled (2 a, 2 l).  Centres in ascending (x, y, z)
    order, each centre's shells in ascending (l, exponents) order; one single-primitive function of
    coefficient 1 per Cartesian component of every am in [0, am_selected] of each cluster (not normalised:
    run normalize_cartesian_basis on the result)."""
    if not orbital_basis:
        raise ValueError("build_auto_auxiliary_basis: empty orbital basis")
    kind = kind.upper()
    if kind not in ("AUTO", "PAUTO"):
        raise ValueError(f"unknown auxiliary basis type '{kind}'")
    centres: dict = {}
    for fn in orbital_basis:
        centres.setdefault((fn.x, fn.y, fn.z), {})[(fn.l, tuple(fn.exponents))] = fn
    aux = []
    for centre in sorted(centres):
        shell_map = centres[centre]
        keys = sorted(shell_map)
        rep = shell_map[keys[0]]
        z = atomic_number(rep.element)
        lmax_obs = max(l for l, _ in keys)
        lmax_abs = max(lmax_obs + lmax_inc, 2 * _lval(z))
        if kind == "PAUTO":
            cands = [(ei + ej, li + lj) for li, ei_list in keys for ei in ei_list for lj, ej_list in keys
                     for ej in ej_list]
        else:
            cands = [(2.0 * e, 2 * l) for l, e_list in keys for e in e_list]
        for e_sel, am_sel in _cluster(cands, f_sam, lmax_abs):
            for am in range(am_sel + 1):
                for c in cartesian_components(am):
                    aux.append(BasisFunction(rep.element, rep.x, rep.y, rep.z, am, c, [e_sel], [1.0]))
    return aux


def flatten(basis: list) -> dict:
    """Plain arrays of a BasisFunction list for the C ABI: center (n, 3), lxyz (n, 3) int32,
    prim_offset (n + 1) int64, exponents and coefficients (concatenated)."""
    n = len(basis)
    center = np.array([[f.x, f.y, f.z] for f in basis], dtype=np.float64).reshape(n, 3)
    lxyz = np.array([f.cartesian for f in basis], dtype=np.int32).reshape(n, 3)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(f.exponents) for f in basis])
    exps = np.array([e for f in basis for e in f.exponents], dtype=np.float64)
    coefs = np.array([c for f in basis for c in f.coefficients], dtype=np.float64)
    for f in basis:
        if sum(f.cartesian) != f.l or len(f.exponents) != len(f.coefficients) or not f.exponents:
            raise ValueError("flatten: inconsistent basis function")
    return dict(center=np.ascontiguousarray(center), lxyz=np.ascontiguousarray(lxyz), prim_offset=off,
                exponents=exps, coefficients=coefs)


def unflatten(d: dict, elements=None) -> list:
    """The inverse of flatten (element names from `elements`, else "X")."""
    out = []
    off = d["prim_offset"]
    for i in range(len(off) - 1):
        c = tuple(int(v) for v in d["lxyz"][i])
        out.append(BasisFunction(elements[i] if elements is not None else "X", float(d["center"][i][0]),
                                 float(d["center"][i][1]), float(d["center"][i][2]), sum(c), c,
                                 [float(v) for v in d["exponents"][off[i]:off[i + 1]]],
                                 [float(v) for v in d["coefficients"][off[i]:off[i + 1]]]))
    return out


def nuclear_repulsion(geometry: list) -> float:
    """sum_{A<B} Z_A Z_B / R_AB (geometry in bohr)."""
    e = 0.0
    for i, a in enumerate(geometry):
        for b in geometry[i + 1:]:
            r = math.sqrt((a.x - b.x) ** 2 + (a.y - b.y) ** 2 + (a.z - b.z) ** 2)
            e += atomic_number(a.symbol) * atomic_number(b.symbol) / r
    return e


def _laplacian(l: int) -> np.ndarray:
    """(n(l-2), n(l)): the Laplacian of each degree-l monomial in degree-(l-2) monomials."""
    src, dst = cartesian_components(l), cartesian_components(l - 2)
    out = np.zeros((len(dst), len(src)))
    for s, (lx, ly, lz) in enumerate(src):
        for d, (a, b, c) in enumerate(((lx - 2, ly, lz), (lx, ly - 2, lz), (lx, ly, lz - 2))):
            if min(a, b, c) >= 0:
                out[dst.index((a, b, c)), s] += (lx, ly, lz)[d] * ((lx, ly, lz)[d] - 1)
    return out


def cartesian_to_spherical_block(l: int) -> np.ndarray:
    """(n(l) x (2l + 1)) block of src/Utils/SphericalTransform.cpp:60-130: the null space of the Laplacian
    on degree-l monomials (eigenvectors of L^T L with zero eigenvalue), Loewdin-orthonormalised in the
    overlap of the normalised Cartesian components (canonical orthogonalisation at 1e-8), expressed in the
    Cartesian components.  The span is unique; the orientation inside it is the eigensolver's."""
    nf, ns = len(cartesian_components(l)), 2 * l + 1
    if nf == ns:
        return np.eye(nf)
    lap = _laplacian(l)
    w, u = np.linalg.eigh(lap.T @ lap)
    null = u[:, :ns]
    comps = cartesian_components(l)
    raw = np.array([[cartesian_self_overlap_pair(l, ci, cj) for cj in comps] for ci in comps])
    d = 1.0 / np.sqrt(np.diag(raw))
    s_norm = raw * d[:, None] * d[None, :]
    m = null.T @ s_norm @ null
    ev, ec = np.linalg.eigh(m)
    keep = ev > 1e-8
    if keep.sum() != ns:
        raise ValueError(f"cartesian_to_spherical_block: l={l}: rank {int(keep.sum())} of {ns}")
    x = ec[:, keep] / np.sqrt(ev[keep])
    if keep.all():
        x = x @ ec.T  # the symmetric form when nothing is dropped, as canonical orthogonalisation gives
    return null @ x


def cartesian_self_overlap_pair(l: int, ci: tuple, cj: tuple, a: float = 1.0) -> float:
    """<x^ci exp(-a r^2) | x^cj exp(-a r^2)> at one centre (unit coefficients, no libcint factor)."""
    v = 1.0
    for p, q in zip(ci, cj):
        k = p + q
        if k % 2:
            return 0.0
        v *= _double_factorial_odd(k // 2) / (4.0 * a) ** (k // 2) * math.sqrt(math.pi / (2.0 * a))
    return v


def build_spherical_transform(functions: list) -> tuple:
    """The block-diagonal Cartesian-to-spherical transform of a normalised Cartesian basis
    (src/Utils/SphericalTransform.cpp:132-165): (T (n_cart x n_sph), [(l, cartesian offset, spherical
    offset)]), shells as consecutive runs of len(cartesian_components(l)) functions."""
    shells, i, n_sph = [], 0, 0
    while i < len(functions):
        l = functions[i].l
        shells.append((l, i, n_sph))
        n_sph += 2 * l + 1
        i += len(cartesian_components(l))
    T = np.zeros((len(functions), n_sph))
    for l, co, so in shells:
        blk = cartesian_to_spherical_block(l)
        T[co:co + blk.shape[0], so:so + blk.shape[1]] = blk
    return T, shells
