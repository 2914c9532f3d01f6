"""Algorithmic FP64 operation counts of the ERI kernels (FMA = 2 flops), per
primitive quartet and per work item of each class, counted from the code the
kernels run.  Used for the roofline of the direct J/K and packed-integral
kernels; cross-checked against ncu's executed dfma/dadd/dmul counts.

Obara--Saika classes (LA+LB+LC+LD = LT <= 4, csrc/os_classes.inc):
  setup     PQ, zeta+eta, 1/sqrt (Newton step), 1/(zeta+eta), T, prefactor: 24
  Boys      counted at the cost of a Taylor evaluation from stored
            coefficients: LT <= 1: grid index and offset 3, Horner 14 (+12 for
            F_1); LT 2, 3: 3 + F_3 Horner 12 + exp series 12 + 2 + recursion
            3 x 3 = 38; LT 4: the same with four recursion steps = 41.  The
            kernels store only {F_top(T_k), exp(-T_k)} per grid point and
            rebuild the coefficients by a downward recursion (about 40 more
            FP64 operations per primitive quartet, in exchange for 48 fewer
            table bytes per lane); that recursion is not counted as
            algorithmic work, so ncu's executed count exceeds this model
  prefactor (LT+1) products
  VRR       the emitted vertical recurrence and the coefficients it reads
            (PA, QC, WP, WQ components, rho/zeta, rho/eta, the 1/(2x) factors;
            gen_os.class_flops)
  per item  the emitted horizontal transfer, plus the J/K digestion
Rys classes (the block-mode classes, 3+ roots):
  roots     NR roots x 2 series (root, weight) x Clenshaw(14 coef): 13 x (FMA+sub)
            + final (FMA+sub)                                     = 84 / root
  setup     T, prefactor: 20
  rys2d     per (root, axis): 12 (coefficients)
            + vertical:  (NB-1) x 3 + (NB+1) x 3 + (NB+1)(MK-1) x 5
            + ket HRR:   (NB+1) x sum_{d=1..LD} (MK-d+1) x 2
            + bra HRR:   (LC+1)(LD+1) x sum_{b=1..LB} (NB-b+1) x 2
  assembly  NAB x NCD x NR x 3   (one MUL + one FMA per component per root)
  where NB = LA+LB, MK = LC+LD, NR = (LA+LB+LC+LD)/2 + 1.
Per work item, the J/K digestion adds NAB x NCD x 16 (weights, six D
products).
"""
from .csrc import gen_os

PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
_OS = set(gen_os.OS_CLASSES)


def ncart(L):
    return (L + 1) * (L + 2) // 2


def quartet_class_ls(qc):
    """(LA, LB, LC, LD) of quartet class index qc = cb(cb+1)/2 + ck."""
    cb = 0
    while (cb + 1) * (cb + 2) // 2 <= qc:
        cb += 1
    ck = qc - cb * (cb + 1) // 2
    return PAIR_CLASSES[cb] + PAIR_CLASSES[ck]


def uses_os(LA, LB, LC, LD):
    return (LA, LB, LC, LD) in _OS


def rys2d_flops(LA, LB, LC, LD):
    NB, MK = LA + LB, LC + LD
    f = 12
    f += max(NB - 1, 0) * 3 + (NB + 1) * 3 * (MK > 0) + (NB + 1) * max(MK - 1, 0) * 5
    f += (NB + 1) * sum((MK - d + 1) * 2 for d in range(1, LD + 1))
    f += (LC + 1) * (LD + 1) * sum((NB - b + 1) * 2 for b in range(1, LB + 1))
    return f


def _os_boys_flops(LT):
    if LT == 0:
        return 3 + 14
    if LT == 1:
        return 3 + 14 + 12
    return 38 if LT <= 3 else 41


def prim_quartet_flops(LA, LB, LC, LD):
    """FP64 flops per primitive quartet of class (LA LB|LC LD)."""
    LT = LA + LB + LC + LD
    if uses_os(LA, LB, LC, LD):
        return 24 + _os_boys_flops(LT) + (LT + 1) + gen_os.class_flops(LA, LB, LC, LD)[0]
    NR = LT // 2 + 1
    nab, ncd = ncart(LA) * ncart(LB), ncart(LC) * ncart(LD)
    return 20 + NR * 84 + NR * 3 * rys2d_flops(LA, LB, LC, LD) + nab * ncd * NR * 3


def digest_flops(LA, LB, LC, LD):
    return ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD) * 16


def item_flops(LA, LB, LC, LD):
    """FP64 flops per work item: the horizontal transfer (Obara--Saika
    classes) and the J/K digestion."""
    hrr = gen_os.class_flops(LA, LB, LC, LD)[1] if uses_os(LA, LB, LC, LD) else 0
    return hrr + digest_flops(LA, LB, LC, LD)


def class_flops(qc, prim_quartets, quartets):
    ls = quartet_class_ls(qc)
    return prim_quartets * prim_quartet_flops(*ls) + quartets * item_flops(*ls)
