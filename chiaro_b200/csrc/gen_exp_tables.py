"""Generate exp_f64_table.inc: 2^(i/128) split into a rounded double H and a
relative tail T = (2^(i/128) - H) / H, stored as (bits(T), bits(H) - (i << 45))
for the table-driven f64 exp in common.cuh. Computed with 80-digit decimals.

Run: python gen_exp_tables.py > exp_f64_table.inc
"""
import struct
from decimal import Decimal, getcontext

getcontext().prec = 80


def bits(x: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def main() -> None:
    print("// Generated by gen_exp_tables.py: 2^(i/128) = H * (1 + T); pairs (bits(T), bits(H) - (i << 45)).")
    print("#define EXP_F64_TABLE_VALUES \\")
    rows = []
    for k in range(128):
        v = Decimal(2) ** (Decimal(k) / Decimal(128))
        h = float(v)
        t = float((v - Decimal(h)) / Decimal(h))
        rows.append("    0x%016xULL, 0x%016xULL" % (bits(t), (bits(h) - (k << 45)) & 0xFFFFFFFFFFFFFFFF))
    print(", \\\n".join(rows))


if __name__ == "__main__":
    main()
