"""Generate the Obara--Saika / Head-Gordon--Pople class routines of the
thread-mode ERI kernels (``os_classes.inc``).

    python -m pyquante_b200.csrc.gen_os            # writes os_classes.inc
    python -m pyquante_b200.csrc.gen_os --count    # op counts, OS vs Rys

For a shell-quartet class (LA LB | LC LD) (LA >= LB, LC >= LD, the pair
orientation of the engine) the scheme of Head-Gordon and Pople (J. Chem.
Phys. 89, 5777 (1988)) -- the scheme of the reference's Src/chgp.c:78-419 --
splits the work in two:

* per primitive quartet, the vertical recurrence of Obara and Saika builds
  the integrals [e0|f0]^(0) for |e| = LA..LA+LB and |f| = LC..LC+LD from
  [00|00]^(m) = K_ab K_cd (zeta+eta)^(-1/2) F_m(T):

    [e+1_i,0|f0]^(m) = PA_i [e0|f0]^(m) + WP_i [e0|f0]^(m+1)
                       + e_i/(2 zeta) ([e-1_i,0|f0]^(m) - rho/zeta [e-1_i,0|f0]^(m+1))
                       + f_i/(2(zeta+eta)) [e0|f-1_i,0]^(m+1)
    [e0|f+1_i,0]^(m) = QC_i [e0|f0]^(m) + WQ_i [e0|f0]^(m+1)
                       + f_i/(2 eta) ([e0|f-1_i,0]^(m) - rho/eta [e0|f-1_i,0]^(m+1))
                       + e_i/(2(zeta+eta)) [e-1_i,0|f0]^(m+1)

  (WP = W - P = -rho/zeta PQ, WQ = W - Q = rho/eta PQ, PQ = P - Q); the
  contraction sums these [e0|f0] over the item's primitive quartets;
* once per work item, the horizontal recurrence moves angular momentum from
  the first centre of each pair to the second on the contracted values,
    (a, b+1_i| = (a+1_i, b| + AB_i (a, b|,   |c, d+1_i) = |c+1_i, d) + CD_i |c, d),
  giving the NAB x NCD components in the order the epilogues read
  (a * NB + b) * NCD + c * ND + d, cartesian components in PyQuante order.

The recursion tree is chosen per class (ket reductions while the ket index
is nonzero; the direction of each step by a greedy search for the fewest new
intermediates, over the six axis preference orders) and written out as
straight-line code, so every index is a constant and every intermediate a
register.  ``--count`` prints the FP64 operations per primitive quartet of
this scheme and of the Rys path (pyquante_b200.flops), from which the class
list below was chosen.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# classes whose thread-mode kernels use the generated routines: every class
# with LA+LB+LC+LD <= 4 (the block-mode classes keep the Rys quadrature)
OS_CLASSES = [(0, 0, 0, 0), (1, 0, 0, 0), (1, 1, 0, 0), (1, 0, 1, 0), (2, 0, 0, 0), (1, 1, 1, 0), (2, 0, 1, 0),
              (2, 1, 0, 0), (1, 1, 1, 1), (2, 0, 1, 1), (2, 0, 2, 0), (2, 1, 1, 0), (2, 2, 0, 0)]


def carts(L):
    """Cartesian components of angular momentum L in PyQuante order
    (PyQuante/Ints.py:23-29): x descending, then y descending."""
    return [(x, y, L - x - y) for x in range(L, -1, -1) for y in range(L - x, -1, -1)]


def _sub(t, i):
    return tuple(v - (1 if j == i else 0) for j, v in enumerate(t))


def _add(t, i):
    return tuple(v + (1 if j == i else 0) for j, v in enumerate(t))


class VRR:
    """Recursion tree of one class: nodes (e, f, m), children by OS."""

    def __init__(self, order):
        self.order = order            # axis preference, e.g. (0, 1, 2)
        self.nodes = {}               # (e, f, m) -> (kind, axis, children)
        self.seq = []                 # topological order

    @staticmethod
    def rule(e, f, m, i):
        """Children of (e, f, m) reduced along axis i (ket if f != 0)."""
        if any(f):
            f1 = _sub(f, i)
            ch = [("X", (e, f1, m)), ("W", (e, f1, m + 1))]
            if f1[i] >= 1:
                f2 = _sub(f1, i)
                ch += [("Y0", (e, f2, m)), ("Y1", (e, f2, m + 1))]
            if e[i] >= 1:
                ch += [("Z", (_sub(e, i), f1, m + 1))]
            return "ket", ch
        e1 = _sub(e, i)
        ch = [("X", (e1, f, m)), ("W", (e1, f, m + 1))]
        if e1[i] >= 1:
            e2 = _sub(e1, i)
            ch += [("Y0", (e2, f, m)), ("Y1", (e2, f, m + 1))]
        return "bra", ch

    def build(self, e, f, m):
        key = (e, f, m)
        if key in self.nodes:
            return
        if not any(e) and not any(f):
            self.nodes[key] = ("base", None, [])
            self.seq.append(key)
            return
        side = f if any(f) else e
        best = None
        for i in (i for i in self.order if side[i] > 0):
            kind, ch = self.rule(e, f, m, i)
            new = sum(1 for _, c in ch if c not in self.nodes)
            if best is None or new < best[0]:
                best = (new, i, kind, ch)
        _, i, kind, ch = best
        for _, c in ch:
            self.build(*c)
        self.nodes[key] = (kind, i, ch)
        self.seq.append(key)


def targets(LA, LB, LC, LD):
    """The accumulated [e0|f0], in the order of the accumulator array."""
    return [(e, f) for le in range(LA, LA + LB + 1) for e in carts(le) for lf in range(LC, LC + LD + 1)
            for f in carts(lf)]


def _term_ops(ch):
    # X*PA (mul) + W*WP (fma) [+ fma for (Y0 - r Y1) + fma] [+ fma for Z]
    names = [n for n, _ in ch]
    return 2 + (2 if "Y0" in names else 0) + (1 if "Z" in names else 0)


def vrr_ops(t):
    """FP64 operations of the VRR per primitive quartet (an FMA is one op)."""
    return sum(_term_ops(t.nodes[k][2]) for k in t.seq if t.nodes[k][0] != "base")


def best_tree(LA, LB, LC, LD):
    best = None
    for order in ((0, 1, 2), (2, 1, 0), (1, 0, 2), (0, 2, 1), (1, 2, 0), (2, 0, 1)):
        t = VRR(order)
        for e, f in targets(LA, LB, LC, LD):
            t.build(e, f, 0)
        ops = vrr_ops(t)
        if best is None or ops < best[0]:
            best = (ops, t)
    return best[1]


def hrr_plan(LA, LB, LC, LD):
    """Straight-line HRR: bra transfers for every ket function f, then ket
    transfers for every final bra pair.  Returns (steps, outputs); a step is
    (dst, hi, lo, axis, 'AB'|'CD'), dst = hi + AB_axis lo."""
    steps = []
    have = set()
    fs = [f for lf in range(LC, LC + LD + 1) for f in carts(lf)]

    def bra(a, b, f):
        if not any(b):
            return ("V", a, f)
        key = ("H", a, b, f)
        if key in have:
            return key
        i = next(j for j in range(3) if b[j] > 0)
        hi = bra(_add(a, i), _sub(b, i), f)
        lo = bra(a, _sub(b, i), f)
        steps.append((key, hi, lo, i, "AB"))
        have.add(key)
        return key

    for a in carts(LA):
        for b in carts(LB):
            for f in fs:
                bra(a, b, f)

    def src(a, b, f):
        return ("V", a, f) if not any(b) else ("H", a, b, f)

    def ket(a, b, c, d):
        if not any(d):
            return src(a, b, c)
        key = ("K", a, b, c, d)
        if key in have:
            return key
        i = next(j for j in range(3) if d[j] > 0)
        hi = ket(a, b, _add(c, i), _sub(d, i))
        lo = ket(a, b, c, _sub(d, i))
        steps.append((key, hi, lo, i, "CD"))
        have.add(key)
        return key

    outs = [ket(a, b, c, d) for a in carts(LA) for b in carts(LB) for c in carts(LC) for d in carts(LD)]
    return steps, outs


def _name(node):
    e, f, m = node
    return "v%d%d%d_%d%d%d_%d" % (e + f + (m,))


def emit_class(LA, LB, LC, LD):
    """C++ source lines of OsClass<LA, LB, LC, LD>, VRR op count, HRR steps."""
    t = best_tree(LA, LB, LC, LD)
    tg = targets(LA, LB, LC, LD)
    tindex = {(e, f): k for k, (e, f) in enumerate(tg)}
    used_by = {}
    for k in t.seq:
        for _, c in t.nodes[k][2]:
            used_by[c] = used_by.get(c, 0) + 1
    L = ["template <> struct OsClass<%d, %d, %d, %d> {" % (LA, LB, LC, LD),
         "    static constexpr bool kOn = true;",
         "    static constexpr int NV = %d;   // accumulated [e0|f0]" % len(tg),
         "    // %d VRR operations per primitive quartet (FMA = 1)" % vrr_ops(t),
         "    template <typename R>",
         "    __device__ static __forceinline__ void vrr(const OsGeom<R> &g, const R *F, R *v)",
         "    {"]
    consts = set()
    body = []
    for k in t.seq:
        kind, i, ch = t.nodes[k]
        e, f, m = k
        nm = _name(k)
        is_target = m == 0 and (e, f) in tindex
        if kind == "base":
            body.append("        const R %s = F[%d];" % (nm, m))
            if is_target:
                body.append("        v[%d] += %s;" % (tindex[(e, f)], nm))
            continue
        d = dict(ch)
        if kind == "bra":
            c1, c2, ki, cy, ry, kz, cz = "g.PA[%d]" % i, "g.WP[%d]" % i, e[i] - 1, "g.oo2z", "g.rz", 0, None
        else:
            c1, c2, ki, cy, ry, kz, cz = "g.QC[%d]" % i, "g.WQ[%d]" % i, f[i] - 1, "g.oo2e", "g.re", e[i], "g.oo2ze"
        if ki > 1:
            consts.add((cy, ki))
            cy = "%s%d" % (cy.replace("g.", "k_"), ki)
        if kz > 1:
            consts.add((cz, kz))
            cz = "%s%d" % (cz.replace("g.", "k_"), kz)
        # a target no other node reads accumulates in place (acc as addend)
        acc = "v[%d]" % tindex[(e, f)] if (is_target and used_by.get(k, 0) == 0) else None
        expr = "fma(%s, %s, %s)" % (c1, _name(d["X"]), acc) if acc else "%s * %s" % (c1, _name(d["X"]))
        expr = "fma(%s, %s, %s)" % (c2, _name(d["W"]), expr)
        if "Y0" in d:
            body.append("        const R %s_y = fma(-%s, %s, %s);" % (nm, ry, _name(d["Y1"]), _name(d["Y0"])))
            expr = "fma(%s, %s_y, %s)" % (cy, nm, expr)
        if "Z" in d:
            expr = "fma(%s, %s, %s)" % (cz, _name(d["Z"]), expr)
        if acc:
            body.append("        %s = %s;" % (acc, expr))
        else:
            body.append("        const R %s = %s;" % (nm, expr))
            if is_target:
                body.append("        v[%d] += %s;" % (tindex[(e, f)], nm))
    for base, k in sorted(consts):
        L.append("        const R %s%d = (R)%d * %s;" % (base.replace("g.", "k_"), k, k, base))
    L += body
    L += ["        (void)F;", "    }"]
    steps, outs = hrr_plan(LA, LB, LC, LD)
    L += ["    template <typename R>",
          "    __device__ static __forceinline__ void hrr(const R *AB, const R *CD, const R *v, R *out)",
          "    {"]

    def ref(s):
        if s[0] == "V":
            return "v[%d]" % tindex[(s[1], s[2])]
        if s[0] == "H":
            return "h_%d%d%d_%d%d%d_%d%d%d" % (s[1] + s[2] + s[3])
        return "k_%d%d%d_%d%d%d_%d%d%d_%d%d%d" % (s[1] + s[2] + s[3] + s[4])

    for dst, hi, lo, i, which in steps:
        L.append("        const R %s = fma(%s[%d], %s, %s);" % (ref(dst), which, i, ref(lo), ref(hi)))
    for k, o in enumerate(outs):
        L.append("        out[%d] = %s;" % (k, ref(o)))
    L += ["        (void)AB;", "        (void)CD;", "    }", "};"]
    return L, vrr_ops(t), len(steps)


def emitted_flops(lines):
    """(vrr, hrr) FP64 flops of the emitted bodies (FMA = 2, MUL/ADD = 1;
    a constant multiple k * coefficient, once per primitive quartet,
    counts 1)."""
    out = {"vrr": 0, "hrr": 0}
    fn = None
    for ln in lines:
        s = ln.strip()
        if "void vrr(" in s:
            fn = "vrr"
            continue
        if "void hrr(" in s:
            fn = "hrr"
            continue
        if fn is None or s.startswith(("template", "static", "//", "(void)")) or "=" not in s:
            continue
        rhs = s.split("=", 1)[1]
        n = 2 * rhs.count("fma(") + rhs.count(" * ") + (1 if "+=" in s else 0)
        out[fn] += n
    return out["vrr"], out["hrr"]


def geometry_flops(lines):
    """Flops of the per-primitive-quartet coefficients the emitted VRR
    reads (the kernel computes the others, but the compiler drops them):
    PA_i, QC_i (a subtraction each), WP_i, WQ_i (a product each, after
    rho/zeta or rho/eta), the three 1/(2x) factors."""
    body = "\n".join(ln for ln in lines if "g." in ln)
    n = sum(1 for f in ("PA", "QC", "WP", "WQ") for i in range(3) if "g.%s[%d]" % (f, i) in body)
    if "g.WP[" in body or "g.rz" in body:
        n += 1
    if "g.WQ[" in body or "g.re" in body:
        n += 1
    n += sum(1 for f in ("oo2z", "oo2e", "oo2ze") if "g.%s" % f in body)
    return n


_FLOPS = {}


def class_flops(LA, LB, LC, LD):
    """Cached (flops per primitive quartet of the VRR and of the coefficients
    it reads, hrr flops per item)."""
    key = (LA, LB, LC, LD)
    if key not in _FLOPS:
        lines = emit_class(*key)[0]
        v, h = emitted_flops(lines)
        _FLOPS[key] = (v + geometry_flops(lines), h)
    return _FLOPS[key]


def as_python(lines):
    """The emitted vrr/hrr bodies as Python functions (a host-side check of
    the generated code itself: the same expressions, FMA as a*b + c)."""
    src, fn = [], None
    for ln in lines:
        s = ln.strip()
        if "void vrr(" in s:
            fn = "vrr"
            src.append("def vrr(g, F, v):")
            continue
        if "void hrr(" in s:
            fn = "hrr"
            src.append("def hrr(AB, CD, v, out):")
            continue
        if fn is None or s in ("{", "}", "};") or s.startswith(("template", "static", "//", "(void)")):
            continue
        s = s.replace("const R ", "").rstrip(";").replace("(R)", "")
        s = re.sub(r"g\.(\w+)", r"g['\1']", s)
        src.append("    " + s)
    env = {"fma": lambda a, b, c: a * b + c}
    exec("\n".join(src), env)
    return env["vrr"], env["hrr"]


def source():
    lines = ["// Generated by gen_os.py -- do not edit.",
             "// Obara--Saika vertical and Head-Gordon--Pople horizontal recurrences per",
             "// class, straight-line (the recurrences are stated in gen_os.py).",
             "#pragma once"]
    report = []
    for cls in OS_CLASSES:
        L, vops, hsteps = emit_class(*cls)
        lines += L
        report.append((cls, vops, hsteps))
    return "\n".join(lines) + "\n", report


def main():
    text, report = source()
    with open(os.path.join(HERE, "os_classes.inc"), "w") as f:
        f.write(text)
    for cls, vops, hsteps in report:
        print("(%d%d|%d%d): VRR %d ops/primitive quartet, HRR %d ops/item" % (cls + (vops, hsteps)))


def count():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from pyquante_b200 import flops
    _saved = flops._OS
    flops._OS = set()          # the Rys model of every class, for comparison
    prim_quartet_flops = flops.prim_quartet_flops
    pairs = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
    for cb in range(6):
        for ck in range(cb + 1):
            cls = pairs[cb] + pairs[ck]
            t = best_tree(*cls)
            steps, _ = hrr_plan(*cls)
            print("(%d%d|%d%d) LT=%d  OS vrr %5d ops (+%d Boys orders) hrr %4d/item   rys model %6d flops" %
                  (cls + (sum(cls), vrr_ops(t), sum(cls) + 1, len(steps), prim_quartet_flops(*cls))))
    flops._OS = _saved


if __name__ == "__main__":
    if "--count" in sys.argv:
        count()
    else:
        main()
