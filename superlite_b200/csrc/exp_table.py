"""Constants of the opacity kernels' table-driven exp (slg_device.cuh).

    python superlite_b200/csrc/exp_table.py

Prints, from 60-digit decimal arithmetic: N/ln2; ln2/N split into a head of
HEAD_BITS significant bits (n * head is exact for |n| < 2^(53 - HEAD_BITS),
which covers |x| <= 700) and the double nearest the remainder; and 2^(j/N),
j = 0..N-1, each the double nearest the exact value.  The header's constants
are this output for N = 64.
"""
import math
from decimal import Decimal, getcontext

N = 64
HEAD_BITS = 36


def constants():
    getcontext().prec = 60
    ln2 = Decimal(2).ln()
    q = ln2 / N
    _, e = math.frexp(float(q))
    scale = Decimal(2) ** (HEAD_BITS - e)
    head = (q * scale).to_integral_value() / scale
    return {"inv_l": float(N / ln2), "l1": float(head), "l2": float(q - head),
            "table": [float(Decimal(2) ** (Decimal(j) / N)) for j in range(N)]}


def main():
    c = constants()
    print(f"kExpInvL = {c['inv_l']!r}  kExpL1 = {c['l1']!r}  kExpL2 = {c['l2']!r}")
    t = c["table"]
    for k in range(0, N, 4):
        print("    " + ", ".join(repr(v) for v in t[k:k + 4]) + ",")


if __name__ == "__main__":
    main()
