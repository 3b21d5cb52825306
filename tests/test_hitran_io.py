"""HITRAN text readers against the reference's own outputs (tests/golden/hitran_golden.npz,
made by tests/golden/make_par_golden.py): every column bit for bit, column lengths
(the reference appends field by field), warnings, errors, and from_files."""

import ctypes
import logging
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN_DIR, ROOT
from pylblrtm_b200 import hitran_io

HIT = os.path.join(GOLDEN_DIR, "hitran")
GOLD = dict(np.load(os.path.join(GOLDEN_DIR, "hitran_golden.npz")))


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and \
        np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("name", ["clean.par", "mixed.par"])
def test_par_to_dict_matches_reference(name, caplog):
    with caplog.at_level(logging.WARNING, logger="pylblrtm_b200.hitran_io"):
        d = hitran_io.par_to_dict(os.path.join(HIT, name))
    assert list(d) == ["nu0", "Sref", "g_air", "g_self", "Elow", "n_air", "shift", "mol_id", "iso_id"]
    for k, v in d.items():
        assert _same(v, GOLD[f"{name}:{k}"]), k
    assert [r.getMessage() for r in caplog.records] == list(GOLD[f"{name}:warnings"])


def test_mixed_file_exercises_the_corner_cases():
    d = hitran_io.par_to_dict(os.path.join(HIT, "mixed.par"))
    lengths = {k: v.size for k, v in d.items()}
    assert len(set(lengths.values())) > 1            # misaligned columns, as the reference
    assert np.isinf(d["Sref"]).sum() == 2 and np.isnan(d["Sref"]).sum() == 1
    assert 1000.5 in d["nu0"]                         # "1_000.5000"


def test_tips_reader_matches_reference():
    t, q = hitran_io.txt_to_tips(os.path.join(HIT, "tips_a.txt"))
    assert _same(t, GOLD["tips_a.txt:T"]) and _same(q, GOLD["tips_a.txt:Q"])


def test_errors_match_reference():
    with pytest.raises(FileNotFoundError, match=r"\.par file not found"):
        hitran_io.par_to_dict(os.path.join(HIT, "missing.par"))
    with pytest.raises(FileNotFoundError, match="TIPS file not found"):
        hitran_io.txt_to_tips(os.path.join(HIT, "missing.txt"))
    with pytest.raises(hitran_io.HITRANDataError, match="No data read"):
        hitran_io.txt_to_tips(os.path.join(HIT, "tips_empty.txt"))
    with pytest.raises(hitran_io.HITRANDataError, match="No valid lines read"):
        hitran_io.par_to_dict(os.path.join(HIT, "tips_empty.txt"))
    assert issubclass(hitran_io.HITRANDataError, ValueError)


def test_from_files(tmp_path):
    d = hitran_io.par_to_dict(os.path.join(HIT, "clean.par"))
    present = sorted(set(zip(d["mol_id"].tolist(), d["iso_id"].tolist())))
    t, q = hitran_io.txt_to_tips(os.path.join(HIT, "tips_a.txt"))
    tips = {k: os.path.join(HIT, "tips_a.txt") for k in present}
    tips[(9, 9)] = (t, q)                             # not in the file: ignored
    sd = hitran_io.from_files(os.path.join(HIT, "clean.par"), tips,
                              molar_masses={k: 18.0 + k[0] for k in present})
    assert sorted(sd.tips) == present and sd.molecule is None
    assert _same(sd.lines["nu0"], d["nu0"])
    with pytest.raises(ValueError, match=re.escape("Missing TIPS for isotopologue(s)")):
        hitran_io.from_files(os.path.join(HIT, "clean.par"), {present[0]: (t, q)}, molar_masses={})


def test_native_reader_counts_universal_newlines():
    lib = hitran_io._lib()
    for text, n in [(b"", 0), (b"a", 1), (b"a\n", 1), (b"a\r\nb", 2), (b"a\rb\n", 2), (b"\n\n", 2), (b"a\r\r\n", 2)]:
        assert lib.lbl_par_count_lines(text, len(text)) == n, text


def test_native_python_float_syntax():
    """The reader's number syntax against Python's float() on a grid of strings."""
    lib = hitran_io._lib()
    cases = ["1", " 1.5 ", "+.5", "-.5", "1.", ".", "", "1e5", "1E-5", "1e", "e5", "1_0", "1__0", "_1", "1_",
             "1_.5", "1._5", "1e1_0", "inf", "-Infinity", "nan", "+NaN", "infin", "0x10", "1d5", "--1", "\t7\x1c",
             "1.5.5", "١"]
    for c in cases:
        if not c.isascii():
            continue
        field = c[:12].rjust(12)
        rec = ("111" + field + "1.000E-20" + " " * 200)[:160]
        raw = rec.encode()
        vals = np.zeros((1, 7))
        ids = np.zeros((1, 2), np.int32)
        st = np.zeros(1, np.int8)
        assert lib.lbl_par_parse(raw, len(raw), 1, vals.ctypes.data, ids.ctypes.data, st.ctypes.data) == 0
        try:
            want = float(field)
        except ValueError:
            want = None
        if want is None:
            assert st[0] == 2, c
        else:
            assert st[0] >= 3, c
            assert np.array_equal(np.float64(want).view(np.uint64), vals[0, 0].view(np.uint64)) or \
                (np.isnan(want) and np.isnan(vals[0, 0])), c
