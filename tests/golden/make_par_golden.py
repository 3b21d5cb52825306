"""Golden vectors for the HITRAN text readers, made by running the REFERENCE's readers.

    python tests/golden/make_par_golden.py --reference <source tree of the reference package>

Writes seeded synthetic ``.par`` and TIPS ``.txt`` files under ``tests/golden/hitran/``
(clean 160-character records with LF endings, and a mixed file with CRLF / CR endings,
short lines, malformed and unusual numbers, Python-float corner cases and non-ASCII
bytes), then reads them with the reference's ``par_to_dict`` / ``txt_to_tips``
(``pylblrtm/hitran_manager.py:816-963``) and stores every column and every logged
warning in ``tests/golden/hitran_golden.npz``.
"""

from __future__ import annotations

import argparse
import logging
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "hitran")


def _fmt_frac(v: float, width: int, dec: int) -> str:
    """Fixed-width decimal without the leading zero when it would not fit."""
    s = f"{v:.{dec}f}"
    if len(s) > width and s.startswith("0."):
        s = s[1:]
    if len(s) > width and s.startswith("-0."):
        s = "-" + s[2:]
    return s[:width].rjust(width)


def record(rng, mol: int, iso: str, nu: float) -> str:
    """One 160-character HITRAN-2004 record with random parameters."""
    s = 10.0 ** rng.uniform(-28, -18)
    a = 10.0 ** rng.uniform(-6, 2)
    rec = (f"{mol:2d}{iso:1s}{nu:12.6f}{s:10.3E}{a:10.3E}"
           f"{_fmt_frac(rng.uniform(0.01, 0.12), 5, 4)}{rng.uniform(0.05, 0.5):5.3f}"
           f"{rng.uniform(0, 5000):10.4f}{_fmt_frac(rng.uniform(-0.3, 0.9), 4, 2)}"
           f"{_fmt_frac(rng.uniform(-0.02, 0.005), 8, 6)}")
    rec += "".join(f"{'q' + str(int(rng.integers(0, 99))):>15s}" for _ in range(4))
    rec += f"{'465432':6s}{'  1  2  3  4':12s} {rng.uniform(1, 50):7.1f}{rng.uniform(1, 50):7.1f}"
    assert len(rec) == 160, len(rec)
    return rec


def write_cases():
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(2024)
    # clean: 3 molecules, LF endings
    lines = []
    for nu in np.sort(rng.uniform(500, 3000, 1000)):
        mol = int(rng.choice([1, 2, 3]))
        lines.append(record(rng, mol, str(int(rng.integers(1, 4))), nu))
    with open(os.path.join(OUT, "clean.par"), "w", newline="") as f:
        f.write("\n".join(lines) + "\n")

    # mixed: every oddity the reader has to reproduce
    base = [record(rng, 1, "1", nu) for nu in np.sort(rng.uniform(1000, 1100, 40))]
    odd = list(base[:10])

    def put(rec, a, b, text):
        text = text.rjust(b - a)[: b - a]
        return rec[:a] + text + rec[b:]

    r = base[10]
    odd.append(put(r, 3, 15, "  1_000.5000"))        # underscores between digits
    odd.append(put(base[11], 3, 15, "  1__00.500 "))  # doubled underscore: malformed
    odd.append(put(base[12], 15, 25, "       inf"))
    odd.append(put(base[13], 15, 25, "      -NaN"))
    odd.append(put(base[14], 15, 25, " 1.234e-25"))
    odd.append(put(base[15], 15, 25, "1.234D-025"))   # Fortran D exponent: malformed
    odd.append(put(base[16], 35, 40, "  .05"))
    odd.append(put(base[17], 55, 59, "+.75"))
    odd.append(put(base[18], 59, 67, "-.004000"))
    odd.append(put(base[19], 59, 67, "        "))     # blank shift: malformed after 8 fields
    odd.append(put(base[20], 2, 3, "A"))              # isotopologue 11 written as 'A'
    odd.append(put(base[21], 0, 2, " x"))
    odd.append(put(base[22], 45, 55, "\t1234.5\t  "))
    odd.append(put(base[23], 3, 15, "1e3"))
    odd.append(put(base[24], 3, 15, "."))
    odd.append(put(base[25], 40, 45, "1_2_3"))
    odd.append(put(base[26], 40, 45, "_123"))
    odd.append(base[27][:155])                        # exactly 155 characters: read
    odd.append(base[28][:154])                        # 154 characters: skipped
    odd.append(base[29][:80])
    odd.append("")
    odd.append(put(base[30], 80, 95, "  café quanta"))        # non-ASCII outside the numbers
    odd.append(put(base[31], 3, 15, "  1050.12é"))            # non-ASCII inside a number
    odd.append(base[32][:100] + "é" * 54)                      # 154 characters once decoded
    odd.append(put(base[33], 0, 2, "+2"))
    odd.append(put(base[34], 15, 25, "  infinity"))
    odd.extend(base[35:])
    text = "\r\n".join(odd[:30]) + "\r" + "\n".join(odd[30:])       # CRLF, a lone CR, then LF
    with open(os.path.join(OUT, "mixed.par"), "wb") as f:
        f.write(text.encode("utf-8") + b"\xff\xfe" + base[0][2:].encode())  # invalid UTF-8, no final newline

    # TIPS tables
    t = np.arange(70.0, 400.0, 1.0)
    with open(os.path.join(OUT, "tips_a.txt"), "w", newline="") as f:
        f.write("# T  Q\r\n\r\n")
        for i, tv in enumerate(t):
            q = 174.0 * (tv / 296.0) ** 1.5
            if i == 5:
                f.write("   75.0\r\n")                # one column: skipped
            if i == 9:
                f.write("   bad  1.0\r\n")            # not a number: skipped
            f.write(f"{tv:8.1f}  {q:14.6f}{'  extra' if i == 7 else ''}\r\n")
    with open(os.path.join(OUT, "tips_empty.txt"), "w") as f:
        f.write("# nothing\n\n")
    return ["clean.par", "mixed.par"], ["tips_a.txt"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    from pylblrtm import hitran_manager as hm
    pars, tips = write_cases()
    msgs = []

    class Catch(logging.Handler):
        def emit(self, rec):
            msgs.append(rec.getMessage())

    logging.getLogger(hm.__name__).addHandler(Catch())
    out = {}
    for name in pars:
        msgs.clear()
        d = hm.par_to_dict(os.path.join(OUT, name))
        for k, v in d.items():
            out[f"{name}:{k}"] = v
        out[f"{name}:warnings"] = np.array(list(msgs), dtype=str)
    for name in tips:
        t, q = hm.txt_to_tips(os.path.join(OUT, name))
        out[f"{name}:T"], out[f"{name}:Q"] = t, q
    np.savez_compressed(os.path.join(HERE, "hitran_golden.npz"), **out)
    print({k: (v.shape, v.dtype) for k, v in out.items()})


if __name__ == "__main__":
    main()
