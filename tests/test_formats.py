"""Text formats of the reference's runs (pfb_formats.h): candidate files and
the master's phase-1 / phase-2 lines (master.c:519-558), host code only."""
import os
import re

import pytest

import pfb200


def _reference_dir():
    """The reference tree the oracle Makefile builds from (REF_DIR)."""
    mk = open(os.path.join(os.path.dirname(__file__), "..", "oracle", "Makefile")).read()
    m = re.search(r"^REF_DIR\s*\?=\s*(\S+)", mk, re.M)
    return os.environ.get("REF_DIR", m.group(1) if m else "")


REF_CANDIDATES = os.path.join(_reference_dir(), "candidatos.txt")


def test_phase_lines_match_the_reference_printf(tmp_path):
    recs = [(50000, 30000, 100, 1, 99, 0), (60, 40, 20, 10, 19, 2), (81, 61, 27, 1, 4, 1), (7, 3, 1, 2, 2, 3)]
    p1, p2 = str(tmp_path / "phase1_survivors.txt"), str(tmp_path / "phase2_primes.txt")
    assert pfb200.write_phase1(p1, recs) == 4
    assert pfb200.write_phase2(p2, recs) == 2
    assert open(p1).read() == "".join("a=%d b=%d c=%d k=%d j=%d\n" % r[:5] for r in recs)
    assert open(p2).read() == ("a=60 b=40 c=20 k=10 j=19 PROBABLE_PRIME_BOTH\n"
                               "a=7 b=3 c=1 k=2 j=2 PRIME\n")
    assert pfb200.write_phase1(p1, recs[:1], append=True) == 1
    assert open(p1).read().count("\n") == 5


def test_candidate_file_round_trip(tmp_path):
    path = str(tmp_path / "cands.txt")
    rows = [(10001, 1334, 249, 25, 91), (50000, 30000, 100, 7, 19), (99991, 12, 7, 9999, 1)]
    with open(path, "w") as f:
        f.write("\n".join(" ".join(map(str, r)) for r in rows) + "\n")
    assert pfb200.read_candidates(path) == rows
    with pytest.raises(pfb200.PfbError):
        pfb200.read_candidates(str(tmp_path / "missing.txt"))


@pytest.mark.skipif(not os.path.exists(REF_CANDIDATES), reason="reference tree absent")
def test_reads_the_reference_candidate_file():
    rows = pfb200.read_candidates(REF_CANDIDATES)
    assert len(rows) == 256 and rows[0] == (10001, 1334, 249, 25, 91)
    assert {r[0] for r in rows} == {10000, 10001, 10010, 10011}
