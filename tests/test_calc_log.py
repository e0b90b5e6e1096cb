"""The convergence log writer against the reference's own log shipped with
its sample model (main/fullwave/MODEL/calc_log/log_g_HDDM_Full_Wave): the
full-wave section rebuilt from its values is the same text."""
import os

import pytest

from adventure_fullwave_b200 import hddm

LOG = os.path.join(os.environ.get("FW_REFERENCE", "/root/reference"), "main", "fullwave", "MODEL", "calc_log",
                   "log_g_HDDM_Full_Wave")


@pytest.mark.skipif(not os.path.exists(LOG), reason="the reference's shipped log is not present")
def test_full_wave_section_matches_the_shipped_log():
    text = open(LOG).read()
    start = text.index("\n\n# Full Wave Analysis") + 1
    section = text[start - 1:]
    lines = section.split("\n")
    total_free = int(lines[3].split()[-1])
    norm0 = float(lines[4].split()[-1])
    hist = [float(l.split()[1]) for l in lines[5:] if l.strip()]
    assert total_free == 20264 and len(hist) == 2566
    assert hddm.calc_log_section(total_free, norm0, hist) == section


@pytest.mark.skipif(not os.path.exists(LOG), reason="the reference's shipped log is not present")
def test_correction_jo_sections_match_the_shipped_log():
    """The two correction-Jo sections at the head of the same log (the
    pre-solve's real and imaginary passes) rebuilt from their values."""
    text = open(LOG).read()
    head = text[:text.index("\n\n# Full Wave Analysis")]
    parts = head.split("\n\n# Correction Jo : ")
    rebuilt = ""
    for chunk, part in zip(parts[1:], ("Real", "Imaginary")):
        lines = chunk.split("\n")
        antenna = int(lines[2].split()[-1])
        total_free = int(lines[3].split()[-1])
        norm0 = float(lines[4].split()[-1])
        hist = [float(l.split()[1]) for l in lines[5:] if l.strip()]
        rebuilt += hddm.correct_jo_log_section(part, antenna, total_free, norm0, hist)
    assert len(parts) == 3
    assert rebuilt == head
