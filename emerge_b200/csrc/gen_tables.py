"""Generator of the closed-form Nedelec-2 (Volakis mixed) element tables.

The reference evaluates the element stiffness K and mass M of every tet with
the 11-point KEAST4 rule (``physics/microwave/assembly/curlcurl.py:277-283``,
``:358-379``). KEAST4 integrates polynomials of degree <= 4 exactly, and every
integrand of this element space is such a polynomial:

* values  N_a = sum_m p_{a,m}(lambda) grad(lambda_m), p of degree <= 2, so
  N_a . N_b has degree <= 4;
* curls   curl N_a = sum_P q_{a,P}(lambda) X_P with X_P = g_i x g_j and q of
  degree <= 1, so curl N_a . curl N_b has degree <= 2.

The quadrature sum therefore equals the exact integral, which we evaluate with
the barycentric monomial rule  int_T l0^a l1^b l2^c l3^d dV =
6 V a! b! c! d! / (a+b+c+d+3)!. For a tet with barycentric gradients g_m
(true gradients, any orientation) and per-tet constant tensors:

    M[x,y] = s_x s_y sum_{m,n} G[m][n] * cM[x][y][m][n],  G[m][n] = (eps g_m).g_n
    K[x,y] = s_x s_y sum_{P,Q} H[P][Q] * cK[x][y][P][Q],  H[P][Q] = (mu^-1 X_P).X_Q

with cM = V * int(p_{x,m} p_{y,n}) / V and cK likewise (exact rationals).
``s_x`` reproduces the reference's orientation convention: it builds
L_m = cofactor_m / |det| (curlcurl.py:142-167, 307-311), i.e. L = sigma * lambda
with sigma = sign(det) in the tet's own vertex order. Basis functions whose
total degree in (L, grad L) is odd (ne2, nf0, nf1) pick up sigma; ne0 does not.

DoFs are numbered in the CANONICAL frame: local vertices relabelled by the rank
of their global node id (the reference orients every edge/face by ascending
global id, optimized.py:262-296), DoF order ne0 e0..e5, ne2 e0..e5, nf0 f0..f3,
nf1 f0..f3 (dofsets.py:39,114-115) with canonical edges
(0,1),(0,2),(0,3),(1,2),(1,3),(2,3) and faces (0,1,2),(0,1,3),(0,2,3),(1,2,3).
Basis definitions follow ccbf.py:537 (_ne0_3d), :569 (_ne2_3d), :790 (_nf0_3d),
:808 (_nf1_3d) and curls :644, :659, :928, :949.

Running this file writes ``nedelec_tables.cuh`` next to it.
"""
from __future__ import annotations

import os
from fractions import Fraction
from math import factorial

EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
FACES = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
PAIR_INDEX = {p: i for i, p in enumerate(EDGES)}

# degree-parity class per canonical DoF: 0 -> ne0 (even), 1 -> odd (carries sigma)
ODD = [0] * 6 + [1] * 6 + [1] * 4 + [1] * 4
# entity index (0..5 edges, 6..9 faces) of each canonical DoF
DOF_ENTITY = list(range(6)) + list(range(6)) + [6 + f for f in range(4)] + [6 + f for f in range(4)]


def _mono(*idx):
    e = [0, 0, 0, 0]
    for i in idx:
        e[i] += 1
    return tuple(e)


def _padd(a, b, s=1):
    out = dict(a)
    for k, v in b.items():
        out[k] = out.get(k, Fraction(0)) + s * v
        if out[k] == 0:
            del out[k]
    return out


def _pmul(a, b):
    out = {}
    for ka, va in a.items():
        for kb, vb in b.items():
            k = tuple(x + y for x, y in zip(ka, kb))
            out[k] = out.get(k, Fraction(0)) + va * vb
    return {k: v for k, v in out.items() if v != 0}


def _lam(i, c=1):
    return {_mono(i): Fraction(c)}


def _const(c):
    return {(0, 0, 0, 0): Fraction(c)}


def _integral_over_v(poly):
    """(1/V) * int_T poly dV for a polynomial in barycentric coordinates."""
    tot = Fraction(0)
    for e, c in poly.items():
        num = 6
        for a in e:
            num *= factorial(a)
        tot += c * Fraction(num, factorial(sum(e) + 3))
    return tot


def _cross(a, b):
    """X term for g_a x g_b -> (pair index, sign)."""
    if a < b:
        return PAIR_INDEX[(a, b)], 1
    return PAIR_INDEX[(b, a)], -1


def basis():
    """Per canonical DoF: (value: {m: poly}, curl: {P: poly})."""
    out = []
    for (i, j) in EDGES:  # ne0 = Li grad Lj - Lj grad Li ; curl = 2 gi x gj
        val = {j: _lam(i), i: _lam(j, -1)}
        curl = {PAIR_INDEX[(i, j)]: _const(2)}
        out.append((val, curl))
    for (i, j) in EDGES:  # ne2 = (Li - Lj)(Li grad Lj - Lj grad Li) ; curl = 3 (Li - Lj) gi x gj
        d = _padd(_lam(i), _lam(j), -1)
        val = {j: _pmul(d, _lam(i)), i: _pmul(d, _lam(j, -1))}
        curl = {PAIR_INDEX[(i, j)]: _pmul(_const(3), d)}
        out.append((val, curl))
    for (i, j, k) in FACES:  # nf0 = Li (Lj grad Lk - Lk grad Lj)
        val = {k: _pmul(_lam(i), _lam(j)), j: _pmul(_lam(i), _lam(k, -1))}
        curl = {}
        for (a, b, poly) in ((i, k, _lam(j)), (i, j, _lam(k, -1)), (j, k, _lam(i, 2))):
            p, s = _cross(a, b)
            curl[p] = _padd(curl.get(p, {}), poly, s)
        out.append((val, curl))
    for (i, j, k) in FACES:  # nf1 = Lj (Li grad Lk - Lk grad Li)
        val = {k: _pmul(_lam(j), _lam(i)), i: _pmul(_lam(j), _lam(k, -1))}
        curl = {}
        for (a, b, poly) in ((j, k, _lam(i)), (j, i, _lam(k, -1)), (i, k, _lam(j, 2))):
            p, s = _cross(a, b)
            curl[p] = _padd(curl.get(p, {}), poly, s)
        out.append((val, curl))
    return out


def tables():
    """Exact tables. Returns (mass_terms, stiff_terms) where each is a dict
    (x, y) -> list of (m, n, Fraction) meaning sum c * T[m][n] for the ordered
    pair (first=x, second=y)."""
    B = basis()
    mass, stiff = {}, {}
    for x in range(20):
        vx, cx = B[x]
        for y in range(20):
            vy, cy = B[y]
            mt = []
            for m, pm in vx.items():
                for n, pn in vy.items():
                    c = _integral_over_v(_pmul(pm, pn))
                    if c != 0:
                        mt.append((m, n, c))
            st = []
            for P, qp in cx.items():
                for Q, qq in cy.items():
                    c = _integral_over_v(_pmul(qp, qq))
                    if c != 0:
                        st.append((P, Q, c))
            mass[(x, y)] = sorted(mt)
            stiff[(x, y)] = sorted(st)
    return mass, stiff


def monomials():
    """All monomials of degree <= 4 in (L0, L1, L2, L3), by degree then
    lexicographically descending exponents."""
    out = []
    for a in range(5):
        for b in range(5 - a):
            for c in range(5 - a - b):
                for d in range(5 - a - b - c):
                    out.append((a, b, c, d))
    return sorted(out, key=lambda e: (sum(e), tuple(-x for x in e)))


MONOS = monomials()
MONO_INDEX = {e: i for i, e in enumerate(MONOS)}


def moment_tables():
    """Quadrature-moment form of the element integrals, for reproducing the
    reference's rounding: with L~ the reference's barycentric values at the 11
    KEAST4 points and mu[alpha] = sum_q w_q L~_q^alpha,

        M[x,y] = V~ sum_(m,n) G~[m][n] * sum_(alpha,c) c * mu[alpha]
        K[x,y] = V~ sum_(P,Q) H~[P][Q] * sum_(alpha,c) c * mu[alpha]

    where the basis polynomials are written in L (no orientation signs:
    L~ and grad L~ already carry them). Returns (mass, stiff): dict (x, y) ->
    list of (a, b, [(monomial index, Fraction c), ...])."""
    B = basis()
    mass, stiff = {}, {}
    for x in range(20):
        vx, cx = B[x]
        for y in range(20):
            vy, cy = B[y]
            mt, st = [], []
            for m, pm in sorted(vx.items()):
                for n, pn in sorted(vy.items()):
                    prod = _pmul(pm, pn)
                    if prod:
                        mt.append((m, n, sorted((MONO_INDEX[e], c) for e, c in prod.items())))
            for P, qp in sorted(cx.items()):
                for Q, qq in sorted(cy.items()):
                    prod = _pmul(qp, qq)
                    if prod:
                        st.append((P, Q, sorted((MONO_INDEX[e], c) for e, c in prod.items())))
            mass[(x, y)] = mt
            stiff[(x, y)] = st
    return mass, stiff


def _fmt(c: Fraction) -> str:
    return f"{float(c)!r}" if c.denominator != 1 else f"{c.numerator}.0"


def emit_header(path: str) -> None:
    """Write one specialisation ``Pair<x, y>`` per ordered canonical pair with
    straight-line multiply-adds (constants as literals), so the element kernel
    needs no table lookups: ``stiff(acc, H)`` adds sum_t c_t * H[P_t][Q_t] and
    ``mass(acc, G)`` adds sum_t c_t * G[m_t][n_t] into ``acc`` through the
    caller-provided ``emg_mac(acc, c, v)``."""
    mass, stiff = tables()
    lines = [
        "// GENERATED by gen_tables.py -- do not edit.",
        "// Closed-form Nedelec-2 (Volakis mixed) element integrals in the canonical",
        "// (vertex-rank) frame: exact barycentric-monomial integrals divided by V.",
        "#pragma once",
        "namespace emg_tables {",
        "// 1 for DoFs whose basis function carries the orientation sign (ne2, nf0, nf1)",
        "__host__ __device__ constexpr int odd(int x) { return x >= 6 ? 1 : 0; }",
        "template <int f, int s> struct Pair;",
    ]
    nterms = 0
    for x in range(20):
        for y in range(20):
            lines.append(f"template <> struct Pair<{x}, {y}> {{")
            body = "".join(f" emg_mac(acc, {_fmt(c)}, H[{a}][{b}]);" for a, b, c in stiff[(x, y)])
            lines.append("  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) {"
                         + body + " }")
            body = "".join(f" emg_mac(acc, {_fmt(c)}, G[{a}][{b}]);" for a, b, c in mass[(x, y)])
            lines.append("  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) {"
                         + body + " }")
            lines.append("};")
            nterms += len(stiff[(x, y)]) + len(mass[(x, y)])
    lines.append(f"// total multiply-adds over the 400 ordered pairs: {nterms}")
    lines.append("}  // namespace emg_tables")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def emit_moment_header(path: str) -> None:
    """Write the quadrature-moment tables: ``emg_moments(L, w, mu)`` adds one
    point's weighted monomials w * L^alpha into mu[70], and ``MPair<x, y>``
    contracts the per-tet tensors with the moments (see moment_tables)."""
    mass, stiff = moment_tables()
    lines = [
        "// GENERATED by gen_tables.py -- do not edit.",
        "// Quadrature-moment form of the Nedelec-2 (Volakis mixed) element integrals:",
        "// entries = sum over tensor terms T[a][b] * (sum_alpha c_alpha * mu[alpha]),",
        "// mu[alpha] = sum_q w_q L_q^alpha over the 11 KEAST4 points.",
        "#pragma once",
        "namespace emg_mtables {",
        f"constexpr int kNumMoments = {len(MONOS)};",
        "template <class R>",
        "__device__ __forceinline__ void emg_moments(const R L[4], R w, R mu[kNumMoments]) {",
    ]
    # build monomials incrementally: degree d from degree d-1 times one L
    name = {}
    for i, e in enumerate(MONOS):
        d = sum(e)
        if d == 0:
            lines.append(f"  const R m{i} = w;")
        else:
            r = max(k for k in range(4) if e[k] > 0)
            prev = list(e)
            prev[r] -= 1
            lines.append(f"  const R m{i} = m{MONO_INDEX[tuple(prev)]} * L[{r}];")
        lines.append(f"  mu[{i}] += m{i};")
        name[e] = i
    lines.append("}")
    lines.append("template <int f, int s> struct MPair;")

    def inner(lst):
        # fixed evaluation order through rounding intrinsics: both triangles of a
        # block then evaluate bitwise identically wherever the code is inlined
        a0, c0 = lst[0]
        e = f"emg_mul({_fmt(c0)}, mu[{a0}])"
        for a, c in lst[1:]:
            e = f"emg_fma({e}, {_fmt(c)}, mu[{a}])"
        return e

    for x in range(20):
        for y in range(20):
            lines.append(f"template <> struct MPair<{x}, {y}> {{")
            body = "".join(f" emg_mac(acc, H[{a}][{b}], {inner(lst)});" for a, b, lst in stiff[(x, y)])
            lines.append("  template <class A, class T, class R> __device__ __forceinline__ static void "
                         "stiff(A &acc, const T &H, const R *mu) {" + body + " }")
            body = "".join(f" emg_mac(acc, G[{a}][{b}], {inner(lst)});" for a, b, lst in mass[(x, y)])
            lines.append("  template <class A, class T, class R> __device__ __forceinline__ static void "
                         "mass(A &acc, const T &G, const R *mu) {" + body + " }")
            lines.append("};")
    lines.append("}  // namespace emg_mtables")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    emit_header(os.path.join(here, "nedelec_tables.cuh"))
    emit_moment_header(os.path.join(here, "nedelec_moment_tables.cuh"))
