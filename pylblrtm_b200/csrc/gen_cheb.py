"""Generate cheb_tables.h: Chebyshev node offsets and DCT weights of the multi-level kernels.

For K = 16 and 8 nodes: node k sits at cos((2k+1) pi / (2K)) of the interval half-width
(float32 values), and coefficient k of the node values f_j is
(2/K) sum_j f_j cos(k (2j+1) pi / (2K)) (float64 weights, row k). The angles are reduced
to [0, 2 pi) in integer arithmetic before the cosine. Run:

    python pylblrtm_b200/csrc/gen_cheb.py > pylblrtm_b200/csrc/cheb_tables.h
"""

import numpy as np


def nodes(k: int):
    return [np.float32(np.cos(np.pi * (2 * i + 1) / (2 * k))) for i in range(k)]


def dct(k: int):
    return [np.cos(np.pi * ((r * (2 * j + 1)) % (4 * k)) / (2 * k)) for r in range(k) for j in range(k)]


def lines(vals, fmt, per):
    out = []
    for i in range(0, len(vals), per):
        tail = ", \\" if i + per < len(vals) else ""
        out.append("    " + ", ".join(fmt(v) for v in vals[i:i + per]) + tail)
    return out


def main():
    print("// Generated by gen_cheb.py: Chebyshev nodes and DCT weights (K = 16 and 8).")
    print("#pragma once")
    for k in (16, 8):
        print(f"// cos((2i+1) pi / {2 * k}), i = 0..{k - 1}")
        print(f"#define LBL_CHEB{k}_NODES \\")
        print("\n".join(lines(nodes(k), lambda v: f"{float(v):.9e}f", 4)))
        print(f"// row r, column j: cos(r (2j+1) pi / {2 * k})")
        print(f"#define LBL_DCT{k} \\")
        print("\n".join(lines(dct(k), lambda v: repr(float(v)), 4)))


if __name__ == "__main__":
    main()
