"""Algorithmic FP operation counts of the ERI kernels (FMA = 2 flops), per
primitive quartet of each class, counted from the loop structure of
csrc/pqb_device.cuh (rys_root, rys2d) and csrc/eri_engine.cuh (assembly).
Used for the roofline of the direct J/K and packed-integral kernels.

  roots     NR roots x 2 series (root, weight) x Clenshaw(14 coef): 13 x (FMA+sub)
            + final (FMA+sub)                                     = 84 / root
  setup     T, prefactor: 20
  rys2d     per (root, axis): 12 (coefficients)
            + vertical:  (NB-1) x 3 + (NB+1) x 3 + (NB+1)(MK-1) x 5
            + ket HRR:   (NB+1) x sum_{d=1..LD} (MK-d+1) x 2
            + bra HRR:   (LC+1)(LD+1) x sum_{b=1..LB} (NB-b+1) x 2
  assembly  NAB x NCD x NR x 3   (one MUL + one FMA per component per root)
where NB = LA+LB, MK = LC+LD, NR = (LA+LB+LC+LD)/2 + 1.
Per shell quartet, the J/K digestion adds NAB x NCD x 16 (scales, six
D products).
"""
PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]


def ncart(L):
    return (L + 1) * (L + 2) // 2


def quartet_class_ls(qc):
    """(LA, LB, LC, LD) of quartet class index qc = cb(cb+1)/2 + ck."""
    cb = 0
    while (cb + 1) * (cb + 2) // 2 <= qc:
        cb += 1
    ck = qc - cb * (cb + 1) // 2
    return PAIR_CLASSES[cb] + PAIR_CLASSES[ck]


def rys2d_flops(LA, LB, LC, LD):
    NB, MK = LA + LB, LC + LD
    f = 12
    f += max(NB - 1, 0) * 3 + (NB + 1) * 3 * (MK > 0) + (NB + 1) * max(MK - 1, 0) * 5
    f += (NB + 1) * sum((MK - d + 1) * 2 for d in range(1, LD + 1))
    f += (LC + 1) * (LD + 1) * sum((NB - b + 1) * 2 for b in range(1, LB + 1))
    return f


def prim_quartet_flops(LA, LB, LC, LD):
    NR = (LA + LB + LC + LD) // 2 + 1
    nab, ncd = ncart(LA) * ncart(LB), ncart(LC) * ncart(LD)
    return 20 + NR * 84 + NR * 3 * rys2d_flops(LA, LB, LC, LD) + nab * ncd * NR * 3


def digest_flops(LA, LB, LC, LD):
    return ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD) * 16


def class_flops(qc, prim_quartets, quartets):
    ls = quartet_class_ls(qc)
    return prim_quartets * prim_quartet_flops(*ls) + quartets * digest_flops(*ls)
