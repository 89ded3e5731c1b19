"""Algorithmic FLOP model of the McMurchie-Davidson J/K quartet kernels.

One fixed count per class (la lb|lc ld), independent of how a kernel
organises the work, used as the numerator of the FP64-pipe roofline:

per primitive quartet (L = la+lb+lc+ld, N3(L) = (L+1)(L+2)(L+3)/6)
  Boys function + prefactor      40 + 3 L
  Hermite R_tuv recursion        3 * sum_{j=1..L} N3(j)
  ket contraction                2 N3(Lab) N3(Lcd) ncart_c ncart_d
  bra contraction                2 N3(Lab) ncart_a ncart_b ncart_c ncart_d
per contracted quartet
  Cartesian -> spherical         2 * (sum over transformed indices of in x out sizes x rest)
  digestion                      2 (2 + 4) n_int   (two Coulomb, four exchange blocks)
"""
from __future__ import annotations


def n3(L: int) -> int:
    return (L + 1) * (L + 2) * (L + 3) // 6


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nsph(l: int, spherical: bool = True) -> int:
    return 2 * l + 1 if (spherical and l >= 2) else ncart(l)


def flops_per_primitive(la, lb, lc, ld) -> float:
    L, lab, lcd = la + lb + lc + ld, la + lb, lc + ld
    boys = 40 + 3 * L
    rtuv = 3 * sum(n3(j) for j in range(1, L + 1))
    ket = 2 * n3(lab) * n3(lcd) * ncart(lc) * ncart(ld)
    bra = 2 * n3(lab) * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    return float(boys + rtuv + ket + bra)


def flops_per_contracted(la, lb, lc, ld, spherical=True) -> float:
    ls = [la, lb, lc, ld]
    dims = [ncart(l) for l in ls]
    sph = 0
    for k, l in enumerate(ls):
        if spherical and l >= 2:
            rest = 1
            for m, d in enumerate(dims):
                if m != k:
                    rest *= d
            sph += 2 * dims[k] * (2 * l + 1) * rest
            dims[k] = 2 * l + 1
    nint = 1
    for l in ls:
        nint *= nsph(l, spherical)
    return float(sph + 2 * 6 * nint)


def class_flops(la, lb, lc, ld, prim_quartets, quartets, spherical=True) -> float:
    return prim_quartets * flops_per_primitive(la, lb, lc, ld) + quartets * flops_per_contracted(la, lb, lc, ld,
                                                                                                   spherical)


# Two-electron gradient (backward kernel), one fixed count per class:
# per primitive quartet the Boys function and R_tuv to L+1, and for each of
# the three differentiated centres (A, B, C; D by translational invariance)
# and each direction the ket and bra contractions with that centre's angular
# momentum raised by one; per contracted quartet the density product (8 flops
# per Cartesian integral) and its contraction with the nine derivative
# blocks (2 flops each).
def grad_flops_per_primitive(la, lb, lc, ld) -> float:
    L = la + lb + lc + ld + 1
    f = 40 + 3 * L + 3 * sum(n3(j) for j in range(1, L + 1))
    for centre in range(3):
        ls = [la, lb, lc, ld]
        ls[centre] += 1
        lab, lcd = ls[0] + ls[1], ls[2] + ls[3]
        ket = 2 * n3(lab) * n3(lcd) * ncart(ls[2]) * ncart(ls[3])
        bra = 2 * n3(lab) * ncart(ls[0]) * ncart(ls[1]) * ncart(ls[2]) * ncart(ls[3])
        f += 3 * (ket + bra)
    return float(f)


def grad_flops_per_contracted(la, lb, lc, ld) -> float:
    ncart4 = ncart(la) * ncart(lb) * ncart(lc) * ncart(ld)
    return float(8 * ncart4 + 2 * 9 * ncart4)


def grad_class_flops(la, lb, lc, ld, prim_quartets, quartets) -> float:
    return prim_quartets * grad_flops_per_primitive(la, lb, lc, ld) + quartets * grad_flops_per_contracted(la, lb, lc,
                                                                                                            ld)
