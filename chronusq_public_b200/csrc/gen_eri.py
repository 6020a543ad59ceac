"""Generate the per-class McMurchie-Davidson ERI device functions.

For every shell-quartet class (la lb | lc ld) with la >= lb, lc >= ld and the bra pair
class not below the ket pair class, this emits one fully unrolled device function

    template <typename T>
    __device__ void eri_<la><lb><lc><ld>(const PrimPair* bra, int nbra,
                                         const PrimPair* ket, int nket,
                                         double3 A, double3 B, double3 C, double3 D,
                                         const double* boys_tab, T* out)

that returns the contracted, normalised (ab|cd) over the reference's basis functions
(spherical for pure shells) in row-major [a][b][c][d] order.  ``boys_tab`` is the
shared-memory Boys table of ``stage_boys<L>`` (eri_common.cuh), L = la+lb+lc+ld.

Method (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978); notation of Helgaker,
Jorgensen & Olsen ch. 9.5 and 9.9):

  (ab|cd) = sum_prims  2 pi^(5/2) / (p q sqrt(p+q)) K_ab K_cd
            sum_tuv E^ab_tuv sum_tau,nu,phi (-1)^(tau+nu+phi) E^cd_tau,nu,phi R_(t+tau,u+nu,v+phi)

The ket Hermite sum is accumulated over ket primitive pairs into W[tuv][cd] for one bra
primitive pair, and the bra Hermite transform is applied once per bra primitive pair.
E coefficients are built per primitive pair by the 1D recursion; R by the standard
downward recursion on n from R^n_000 = (-2 rho)^n F_n(rho |PQ|^2).  Boys values come
from :file:`boys.cuh` in FP64 regardless of ``T``; everything after them runs in ``T``.

Run:  python gen_eri.py <out.cuh> [maxl]
"""
import itertools
import os
import sys
from math import comb, sqrt, floor

import numpy as np


def cart_list(l):
    out = []
    for i in range(l + 1):
        for j in range(i + 1):
            out.append((l - i, i - j, j))
    return out


def herm_list(n):
    """(t,u,v) with t+u+v <= n, ordered by total then CCA order."""
    out = []
    for L in range(n + 1):
        out.extend(cart_list(L))
    return out


def _dfact(n):
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def solid_harmonic_matrix(l):
    """Rows m=-l..l of unit-normalised real solid harmonics (x^l-normalised Cartesians).
    Same construction as chronusq_public_b200.basis.solid_harmonic_matrix (Helgaker eqs.
    6.4.47-6.4.50), duplicated so the generator has no package import."""
    carts = cart_list(l)
    idx = {c: k for k, c in enumerate(carts)}
    mat = np.zeros((2 * l + 1, len(carts)))
    for m in range(-l, l + 1):
        am = abs(m)
        vm = 0.0 if m >= 0 else 0.5
        row = np.zeros(len(carts))
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                nv = int(floor(am / 2.0 - vm))
                for iv in range(nv + 1):
                    v = iv + vm
                    two_v = int(round(2 * v))
                    sign = (-1.0) ** int(round(t + v - vm))
                    c = (sign * 0.25 ** t * comb(l, t) * comb(l - t, am + t) * comb(t, u) * comb(am, two_v))
                    row[idx[(2 * t + am - 2 * u - two_v, 2 * u + two_v, l - 2 * t - am)]] += c
        gram = np.zeros((len(carts), len(carts)))
        for a, (ax, ay, az) in enumerate(carts):
            for b, (bx, by, bz) in enumerate(carts):
                sx, sy, sz = ax + bx, ay + by, az + bz
                if sx % 2 or sy % 2 or sz % 2:
                    continue
                gram[a, b] = _dfact(sx - 1) * _dfact(sy - 1) * _dfact(sz - 1) / _dfact(2 * l - 1)
        mat[m + l] = row / sqrt(float(row @ gram @ row))
    return mat


def lit(x):
    r = repr(float(x))
    return "T(%s)" % r


class Gen:
    def __init__(self):
        self.lines = []
        self.ind = 1

    def w(self, s):
        self.lines.append("  " * self.ind + s)


def emit_E(g, tag, la, lb, need):
    """Emit 1D Hermite coefficients E{tag}{dir}_{i}_{j}_{t} for dir in x,y,z.
    Variables used: {tag}PA{d}, {tag}PB{d}, {tag}o2p (=1/(2p)).  Only (i,j) in `need[d]`
    plus their recursion predecessors are emitted."""
    names = {}
    for d in "xyz":
        # closure of needed (i,j)
        req = set()
        stack = list(need[d])
        while stack:
            ij = stack.pop()
            if ij in req:
                continue
            req.add(ij)
            i, j = ij
            if i > 0:
                stack.append((i - 1, j))
            elif j > 0:
                stack.append((i, j - 1))
        order = sorted(req, key=lambda x: (x[0] + x[1], x[0]))
        for (i, j) in order:
            for t in range(i + j + 1):
                nm = "E%s%s_%d_%d_%d" % (tag, d, i, j, t)
                names[(d, i, j, t)] = nm
                if i == 0 and j == 0:
                    continue  # E_0_0_0 = 1 handled symbolically
                if i > 0:
                    pi, pj, X = i - 1, j, "%sPA%s" % (tag, d)
                else:
                    pi, pj, X = i, j - 1, "%sPB%s" % (tag, d)
                terms = []

                def ref(tt):
                    if tt < 0 or tt > pi + pj:
                        return None
                    if pi == 0 and pj == 0:
                        return "T(1)" if tt == 0 else None
                    return "E%s%s_%d_%d_%d" % (tag, d, pi, pj, tt)
                a = ref(t - 1)
                if a:
                    terms.append("%so2p * %s" % (tag, a) if a != "T(1)" else "%so2p" % tag)
                b = ref(t)
                if b:
                    terms.append("%s * %s" % (X, b) if b != "T(1)" else X)
                c = ref(t + 1)
                if c:
                    terms.append("T(%d) * %s" % (t + 1, c) if t + 1 > 1 else c)
                g.w("const T %s = %s;" % (nm, " + ".join(terms) if terms else "T(0)"))
    return names


def Ename(tag, d, i, j, t):
    if i == 0 and j == 0:
        return None  # equals 1
    return "E%s%s_%d_%d_%d" % (tag, d, i, j, t)


def herm_terms(tag, ca, cb):
    """List of ((t,u,v), [factor names]) for the Hermite expansion of Cartesian pair."""
    out = []
    rngs = [range(ca[k] + cb[k] + 1) for k in range(3)]
    for t in rngs[0]:
        for u in rngs[1]:
            for v in rngs[2]:
                fac = []
                for d, (i, j, tt) in zip("xyz", ((ca[0], cb[0], t), (ca[1], cb[1], u), (ca[2], cb[2], v))):
                    nm = Ename(tag, d, i, j, tt)
                    if nm:
                        fac.append(nm)
                out.append(((t, u, v), fac))
    return out


def _wname(members, j, m, h, c):
    return "W%d_%d_%d_%d" % (j, m, h, c) if members else "W%d_%d_%d" % (j, h, c)


def _aname(members, mb, mk, i):
    return "acc%d_%d_%d" % (mb, mk, i) if members else "acc%d" % i


def _emit_tile(g, nbt, la, lb, lc, ld, ca, cb, cc, cd, hp, hidx, ncd, members=None, nkt=1, prefetch=True):
    """One pass over `nbt` bra primitive pairs starting at bra[ib]: their E coefficients,
    the ket loop (each ket primitive pair loaded and its E coefficients built once for
    all nbt bra primitives; with nkt > 1, nkt ket primitive pairs per iteration, whose
    Boys / R chains are independent, then a one-at-a-time remainder), and the bra
    transforms into acc.

    members = (mb, mk) emits the sibling form: the primitive pairs carry unit contraction
    coefficients, bw[m * nbra + i] / kw[m * nket + i] are member m's coefficient products,
    and one W per ket member and one acc per (bra member, ket member) are accumulated from
    the same primitive integrals."""
    L = la + lb + lc + ld
    mb, mk = members if members else (1, 1)
    needb = {d: set() for d in "xyz"}
    for a in ca:
        for b in cb:
            for k, d in enumerate("xyz"):
                needb[d].add((a[k], b[k]))
    for j in range(nbt):
        bt = "b%d" % j
        g.w("const PrimPair pb%d = bra[ib + %d];" % (j, j))
        g.w("const double p%d = pb%d.p;" % (j, j))
        g.w("const T %so2p = T(0.5 * pb%d.ip);" % (bt, j))
        for d in "xyz":
            g.w("const T %sPA%s = T(pb%d.P%s - A.%s);" % (bt, d, j, d, d))
            g.w("const T %sPB%s = T(pb%d.P%s - B.%s);" % (bt, d, j, d, d))
        emit_E(g, bt, la, lb, needb)
        for m in range(mk):
            for h in range(len(hp)):
                for c in range(ncd):
                    g.w("T %s = T(0);" % _wname(members, j, m, h, c))
    needk = {d: set() for d in "xyz"}
    for c in cc:
        for dd in cd:
            for k, d in enumerate("xyz"):
                needk[d].add((c[k], dd[k]))

    def ket_quantities(ktag, qname, kcp):
        """Ket primitive pair p<ktag>: its exponent, E coefficients and the signed ket
        Hermite coefficients kc (shared by the nbt bra primitives)."""
        g.w("const double %s = p%s.p;" % (qname, ktag))
        g.w("const T %so2p = T(0.5 * p%s.ip);" % (ktag, ktag))
        if members:
            for m in range(mk):
                g.w("const T kw%d = T(kw[%d * nket + ik]);" % (m, m))
        for d in "xyz":
            g.w("const T %sPA%s = T(p%s.P%s - C.%s);" % (ktag, d, ktag, d, d))
            g.w("const T %sPB%s = T(p%s.P%s - D.%s);" % (ktag, d, ktag, d, d))
        emit_E(g, ktag, lc, ld, needk)
        kterms = []
        ci = 0
        for c in cc:
            for dd in cd:
                for (tnp, fac) in herm_terms(ktag, c, dd):
                    sgn = -1 if (sum(tnp) % 2) else 1
                    coef = " * ".join(fac) if fac else None
                    cname = "%s%d_%d_%d_%d" % (kcp, ci, tnp[0], tnp[1], tnp[2])
                    cexpr = ("T(%d)" % sgn) if coef is None else (("-" if sgn < 0 else "") + "(" + coef + ")")
                    g.w("const T %s = %s;" % (cname, cexpr))
                    kterms.append((ci, tnp, cname))
                ci += 1
        return kterms

    def chain(j, ktag, qname, kterms, r):
        """One primitive quartet (bra primitive j, ket primitive p<ktag>): Boys values, the R
        recursion and the ket transform into W."""
        g.w("{")
        g.ind += 1
        g.w("const double pq = p%d + %s;" % (j, qname))
        g.w("const double rpq = rsqrt(pq);")
        g.w("const double rho = p%d * %s * (rpq * rpq);" % (j, qname))
        g.w("const double PQx = pb%d.Px - p%s.Px, PQy = pb%d.Py - p%s.Py, PQz = pb%d.Pz - p%s.Pz;"
            % (j, ktag, j, ktag, j, ktag))
        g.w("const double Tb = rho * (PQx * PQx + PQy * PQy + PQz * PQz);")
        g.w("double F[%d];" % (L + 1))
        g.w("boys_eval_sm<%d>(Tb, boys_tab, F);" % L)
        g.w("double fac = pb%d.Kp * p%s.Kp * rpq;" % (j, ktag))
        if L > 0:
            g.w("const double m2r = -2.0 * rho;")
        for n in range(L + 1):
            g.w("const T %s%d_0_0_0 = T(fac * F[%d]);" % (r, n, n))
            if n < L:
                g.w("fac *= m2r;")
        if L > 0:
            g.w("const T Xpq = T(PQx), Ypq = T(PQy), Zpq = T(PQz);")
        for n in range(L - 1, -1, -1):
            for tot in range(1, L - n + 1):
                for (t, u, v) in cart_list(tot):
                    if t > 0:
                        a = "%s%d_%d_%d_%d" % (r, n + 1, t - 1, u, v)
                        b = ("%s%d_%d_%d_%d" % (r, n + 1, t - 2, u, v)) if t > 1 else None
                        expr = "Xpq * %s" % a + ((" + T(%d) * %s" % (t - 1, b)) if b else "")
                    elif u > 0:
                        a = "%s%d_%d_%d_%d" % (r, n + 1, t, u - 1, v)
                        b = ("%s%d_%d_%d_%d" % (r, n + 1, t, u - 2, v)) if u > 1 else None
                        expr = "Ypq * %s" % a + ((" + T(%d) * %s" % (u - 1, b)) if b else "")
                    else:
                        a = "%s%d_%d_%d_%d" % (r, n + 1, t, u, v - 1)
                        b = ("%s%d_%d_%d_%d" % (r, n + 1, t, u, v - 2)) if v > 1 else None
                        expr = "Zpq * %s" % a + ((" + T(%d) * %s" % (v - 1, b)) if b else "")
                    g.w("const T %s%d_%d_%d_%d = %s;" % (r, n, t, u, v, expr))
        # ket transform: W[tuv][cd] += sum_{tau nu phi} (-1)^(..) Ecd * R0_{t+tau,...}
        if not members:
            for (ci, tnp, cname) in kterms:
                for hi, (t, u, v) in enumerate(hp):
                    g.w("W%d_%d_%d += %s * %s0_%d_%d_%d;" % (j, hi, ci, cname, r, t + tnp[0], u + tnp[1], v + tnp[2]))
        else:
            # the ket sum once per (tuv, cd), then one weighted update per ket member
            for ci in range(ncd):
                terms = [(tnp, cname) for (cj, tnp, cname) in kterms if cj == ci]
                for hi, (t, u, v) in enumerate(hp):
                    expr = " + ".join("%s * %s0_%d_%d_%d" % (cname, r, t + tnp[0], u + tnp[1], v + tnp[2])
                                      for (tnp, cname) in terms)
                    g.w("{ const T ks = %s;" % expr)
                    for m in range(mk):
                        g.w("  %s += kw%d * ks;" % (_wname(members, j, m, hi, ci), m))
                    g.w("}")
        g.ind -= 1
        g.w("}")

    if nkt > 1 and not members:
        # ket primitive pairs nkt at a time: nkt independent Boys / R chains per bra primitive
        g.w("int ik = 0;")
        g.w("for (; ik + %d < nket; ik += %d) {" % (nkt - 1, nkt))
        g.ind += 1
        tiles = []
        for m in range(nkt):
            g.w("const PrimPair pk%d = ket[ik + %d];" % (m, m))
        for m in range(nkt):
            tiles.append(ket_quantities("k%d" % m, "qk%d" % m, "kc%d_" % m))
        for j in range(nbt):
            for m in range(nkt):
                chain(j, "k%d" % m, "qk%d" % m, tiles[m], "r%dk%d_" % (j, m))
        g.ind -= 1
        g.w("}")
        g.w("PrimPair pk_next;")
        g.w("if (ik < nket) pk_next = ket[ik];")
        g.w("for (; ik < nket; ++ik) {")
    elif prefetch:
        g.w("PrimPair pk_next;")
        g.w("if (nket > 0) pk_next = ket[0];")
        g.w("for (int ik = 0; ik < nket; ++ik) {")
    else:
        g.w("for (int ik = 0; ik < nket; ++ik) {")
    g.ind += 1
    if prefetch or nkt > 1:
        g.w("const PrimPair pk = pk_next;")
        g.w("if (ik + 1 < nket) pk_next = ket[ik + 1];")
    else:
        g.w("const PrimPair pk = ket[ik];")
    kterms = ket_quantities("k", "q", "kc_")
    for j in range(nbt):
        chain(j, "k", "q", kterms, "r%d_" % j)
    g.ind -= 1
    g.w("}")
    # bra transform: acc[ab][cd] += sum_tuv Eab_tuv W[tuv][cd]
    for j in range(nbt):
        if members:
            for m in range(mb):
                g.w("const T bw%d_%d = T(bw[%d * nbra + ib + %d]);" % (j, m, m, j))
        ai = 0
        for a in ca:
            for b in cb:
                for (tuv, fac) in herm_terms("b%d" % j, a, b):
                    hi = hidx[tuv]
                    coef = " * ".join(fac) if fac else "T(1)"
                    g.w("{ const T bc = %s;" % coef)
                    if not members:
                        for c in range(ncd):
                            g.w("  acc%d += bc * W%d_%d_%d;" % (ai * ncd + c, j, hi, c))
                    else:
                        for m1 in range(mb):
                            g.w("  { const T bcw = bc * bw%d_%d;" % (j, m1))
                            for m2 in range(mk):
                                for c in range(ncd):
                                    g.w("    %s += bcw * %s;" % (_aname(members, m1, m2, ai * ncd + c),
                                                                _wname(members, j, m2, hi, c)))
                            g.w("  }")
                    g.w("}")
                ai += 1


def gen_class(la, lb, lc, ld, pa, pb, pc, pd, nbt=1, members=None, nkt=1, prefetch=True):
    """Device function of one class; nbt > 1 walks the bra primitive pairs nbt at a time
    (each ket primitive pair is then read once per nbt bra primitives), with a one-at-a-time
    loop for the remainder.  prefetch loads the next ket primitive pair one step ahead.

    members = (mb, mk) emits eri_gc_<class>_<mb>x<mk> instead: mb bra and mk ket sibling
    pairs (same centres, angular momenta and exponents, different contraction coefficients)
    evaluated from one set of primitive integrals.  Its arguments add the coefficient
    products bw (mb x nbra) and kw (mk x nket) after bra and ket, whose PrimPair Kp carry unit
    coefficients; out holds mb * mk quartets, member (i, j) at out + (i * mk + j) * n."""
    p_l = la + lb
    ca, cb, cc, cd = cart_list(la), cart_list(lb), cart_list(lc), cart_list(ld)
    nab, ncd = len(ca) * len(cb), len(cc) * len(cd)
    hp = herm_list(p_l)
    hidx = {h: k for k, h in enumerate(hp)}
    mb, mk = members if members else (1, 1)
    g = Gen()
    g.lines.append("template <typename T>")
    if not members:
        name = "eri_%d%d%d%d" % (la, lb, lc, ld)
        g.lines.append("__device__ __forceinline__ void %s(const PrimPair* __restrict__ bra, int nbra,"
                       " const PrimPair* __restrict__ ket, int nket, double3 A, double3 B, double3 C,"
                       " double3 D, const double* __restrict__ boys_tab, T* __restrict__ out) {" % name)
    else:
        name = "eri_gc_%d%d%d%d_%dx%d" % (la, lb, lc, ld, mb, mk)
        g.lines.append("__device__ __forceinline__ void %s(const PrimPair* __restrict__ bra,"
                       " const double* __restrict__ bw, int nbra, const PrimPair* __restrict__ ket,"
                       " const double* __restrict__ kw, int nket, double3 A, double3 B, double3 C,"
                       " double3 D, const double* __restrict__ boys_tab, T* __restrict__ out) {" % name)
    for m1 in range(mb):
        for m2 in range(mk):
            for i in range(nab * ncd):
                g.w("T %s = T(0);" % _aname(members, m1, m2, i))
    g.w("int ib = 0;")
    if nbt > 1:
        g.w("for (; ib + %d < nbra; ib += %d) {" % (nbt - 1, nbt))
        g.ind += 1
        _emit_tile(g, nbt, la, lb, lc, ld, ca, cb, cc, cd, hp, hidx, ncd, members, nkt, prefetch)
        g.ind -= 1
        g.w("}")
    g.w("for (; ib < nbra; ++ib) {")
    g.ind += 1
    _emit_tile(g, 1, la, lb, lc, ld, ca, cb, cc, cd, hp, hidx, ncd, members, nkt, prefetch)
    g.ind -= 1
    g.w("}")
    # spherical transform, axis by axis: cart arrays named by index tuples
    pures = [pa, pb, pc, pd]
    ls = [la, lb, lc, ld]
    for m1 in range(mb):
        for m2 in range(mk):
            dims = [len(ca), len(cb), len(cc), len(cd)]
            pre = "m%d_%d_" % (m1, m2) if members else ""
            cur = {}
            for idx in itertools.product(*[range(x) for x in dims]):
                flat = ((idx[0] * dims[1] + idx[1]) * dims[2] + idx[2]) * dims[3] + idx[3]
                cur[idx] = _aname(members, m1, m2, flat)
            stage = 0
            for ax in range(4):
                if not pures[ax]:
                    continue
                M = solid_harmonic_matrix(ls[ax])
                ns = 2 * ls[ax] + 1
                newdims = list(dims)
                newdims[ax] = ns
                new = {}
                for idx in itertools.product(*[range(x) for x in newdims]):
                    terms = []
                    for k in range(dims[ax]):
                        cval = M[idx[ax], k]
                        if abs(cval) < 1e-15:
                            continue
                        src = list(idx)
                        src[ax] = k
                        terms.append("%s * %s" % (lit(cval), cur[tuple(src)]))
                    nm = "%ss%d_%s" % (pre, stage, "_".join(map(str, idx)))
                    g.w("const T %s = %s;" % (nm, " + ".join(terms) if terms else "T(0)"))
                    new[idx] = nm
                cur = new
                dims = newdims
                stage += 1
            nout = dims[0] * dims[1] * dims[2] * dims[3]
            base = (m1 * mk + m2) * nout
            for idx in itertools.product(*[range(x) for x in dims]):
                flat = ((idx[0] * dims[1] + idx[1]) * dims[2] + idx[2]) * dims[3] + idx[3]
                g.w("out[%d] = %s;" % (base + flat, cur[idx]))
    g.lines.append("}")
    return name, "\n".join(g.lines)


def pair_classes(maxl):
    return [(a, b) for a in range(maxl + 1) for b in range(a + 1)]


def quartet_classes(maxl):
    pcs = pair_classes(maxl)
    out = []
    for i, P in enumerate(pcs):
        for j, Qc in enumerate(pcs):
            if j <= i:
                out.append((P[0], P[1], Qc[0], Qc[1]))
    return out


# classes evaluated by the warp-cooperative kernel (eri_warp.cuh): their Cartesian output
# ncart(a)ncart(b)ncart(c)ncart(d) exceeds 150 values or whose R_tuv set (L >= 6, 84+ values)
# is too large for one thread's registers
def _nc(l):
    return (l + 1) * (l + 2) // 2


WARP_CLASSES = {q for q in quartet_classes(3)
                if _nc(q[0]) * _nc(q[1]) * _nc(q[2]) * _nc(q[3]) > 150 or sum(q) >= 6}


# classes whose bra primitive pairs are walked several at a time, so that each ket
# primitive pair read serves several primitive quartets.  Measured on (H2O)_32 cc-pVDZ:
# (ss|ss) 12.3 -> 8.1 ms with 4 at a time (8: 12 % slower); (ps|ss) 12.85 -> 10.05 ms with 3
# (156 registers, three CTAs per SM; 2: 10.58, 4: 11.42 ms).  (ps|ps), (pp|ss), (ds|ss),
# (dp|ss) get 6-29 % slower with 2 (register pressure), so they keep one.
BRA_TILE = {(0, 0, 0, 0): 4, (1, 0, 0, 0): 3}
# the same for the sibling forms (members_header), whose member accumulators leave less room:
# (ps|ss) 2 x 4 with three bra primitives at a time reaches 255 registers and spills
GC_BRA_TILE = {(0, 0, 0, 0): 4}

# classes whose ket primitive pairs are walked several at a time within each bra primitive
# (independent chains of Boys values and R recursion per iteration).  Measured on (H2O)_32
# cc-pVDZ and rejected: two ket primitives per iteration made (ps|ss), (ps|ps), (pp|ss),
# (ds|ss), (pp|ps), (ds|ps) 5-11 % slower, and (ss|ss) with 2 bra x 2 ket instead of 4 bra
# 18 % slower; so no class uses it.
KET_TILE = {}

# classes whose ket loop loads each primitive pair where it is used instead of one step
# ahead.  Measured on (H2O)_32 cc-pVDZ with every per-thread class both ways: the prefetch
# is worth 0.2-0.45 ms per class on the s and p classes ((ps|ss) 13.04 against 13.48 ms even
# though the variant without it fits five CTAs per SM instead of four), and costs 0.03-0.13
# ms on these, the spilling classes among them.
NO_KET_PREFETCH = {(1, 1, 1, 1), (2, 0, 0, 0), (2, 0, 1, 1), (2, 0, 2, 0), (2, 1, 2, 0), (2, 2, 1, 0)}


# Sibling-group classes of the engine (la, lb, lc, ld, mb, mk): their lists hold entries of
# one bra and one ket group of sibling pairs (same centres, angular momenta and exponents),
# evaluated from one set of primitive integrals with mb bra and mk ket member weights.  mb
# and mk are the member caps of the bra and ket pair classes (s-s pairs 4, p-s and d-s 2,
# p-p 1; csrc/engine_impl.cuh, sibling_cap); the classes are the per-thread ones whose
# sibling form stays within the register file.
GROUP_SPECS = [(0, 0, 0, 0, 4, 4), (1, 0, 0, 0, 2, 4), (1, 0, 1, 0, 2, 2), (1, 1, 0, 0, 1, 4),
               (2, 0, 0, 0, 2, 4)]


def members_header(specs):
    """Header text with the sibling-member variants for `specs` = [(la, lb, lc, ld, mb, mk)],
    each behind EriClassGC<la, lb, lc, ld, mb, mk>::run, the list macro CQG_GC_LIST and the
    per-spec macro CQG_GC_EACH."""
    parts = ["// GENERATED by gen_eri.py (sibling-member variants) -- do not edit.",
             "#pragma once",
             "#include \"../eri_common.cuh\"",
             "template <int LA, int LB, int LC, int LD, int MB, int MK> struct EriClassGC;",
             ""]
    for (la, lb, lc, ld, mb, mk) in specs:
        name, code = gen_class(la, lb, lc, ld, la > 1, lb > 1, lc > 1, ld > 1,
                               nbt=GC_BRA_TILE.get((la, lb, lc, ld), 1), members=(mb, mk))
        parts.append(code)
        parts.append("template <> struct EriClassGC<%d, %d, %d, %d, %d, %d> {" % (la, lb, lc, ld, mb, mk))
        parts.append("  template <typename T> static __device__ __forceinline__ void run(const PrimPair* bra,"
                     " const double* bw, int nbra, const PrimPair* ket, const double* kw, int nket, double3 A,"
                     " double3 B, double3 C, double3 D, const double* boys_tab, T* out) {")
        parts.append("    %s<T>(bra, bw, nbra, ket, kw, nket, A, B, C, D, boys_tab, out);" % name)
        parts.append("  }")
        parts.append("};")
        parts.append("")
    parts.append("#define CQG_GC_LIST(X) {" + ", ".join("X(%d, %d, %d, %d, %d, %d)" % q for q in specs) + "}")
    parts.append("#define CQG_GC_EACH(X) " + " ".join("X(%d, %d, %d, %d, %d, %d)" % q for q in specs))
    return "\n".join(parts) + "\n"


def main(path, maxl=2):
    parts = ["// GENERATED by gen_eri.py -- do not edit.",
             "#pragma once",
             "#include \"../eri_common.cuh\"",
             ""]
    for l in (2, 3):
        M = solid_harmonic_matrix(l)
        parts.append("__constant__ double kSph%d[%d] = {%s};" % (l, M.size, ", ".join(repr(float(x)) for x in M.ravel())))
    parts.append("")
    for (la, lb, lc, ld) in quartet_classes(maxl):
        if (la, lb, lc, ld) in WARP_CLASSES:
            continue
        _, code = gen_class(la, lb, lc, ld, la > 1, lb > 1, lc > 1, ld > 1,
                            nbt=BRA_TILE.get((la, lb, lc, ld), 1), nkt=KET_TILE.get((la, lb, lc, ld), 1),
                            prefetch=(la, lb, lc, ld) not in NO_KET_PREFETCH)
        parts.append(code)
        parts.append("template <> struct EriClass<%d, %d, %d, %d> {" % (la, lb, lc, ld))
        parts.append("  template <typename T> static __device__ __forceinline__ void run(const PrimPair* bra, int nbra,"
                     " const PrimPair* ket, int nket, double3 A, double3 B, double3 C, double3 D,"
                     " const double* boys_tab, T* out) {")
        parts.append("    eri_%d%d%d%d<T>(bra, nbra, ket, nket, A, B, C, D, boys_tab, out);" % (la, lb, lc, ld))
        parts.append("  }")
        parts.append("};")
        parts.append("")
    qcs = quartet_classes(maxl)
    parts.append("// quartet classes in engine order (bra pair class >= ket pair class)")
    parts.append("#define CQG_CLASS_LIST(X, T) \\")
    parts.append("  {" + ", ".join("X(%d, %d, %d, %d, T)" % q for q in qcs) + "}")
    parts.append("#define CQG_GEN_MAXL %d" % maxl)
    parts.append("")
    with open(path, "w") as f:
        f.write("\n".join(parts))
    with open(os.path.join(os.path.dirname(os.path.abspath(path)), "eri_gc_classes.cuh"), "w") as f:
        f.write(members_header([q for q in GROUP_SPECS if max(q[:4]) <= maxl]))


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 2)
