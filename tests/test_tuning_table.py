"""The tile-plan table the autotuner writes and libsynx reads (host logic, no GPU): parsing,
skipping of malformed lines, and the committed table's format."""
import os

from ants_b200 import synx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_table_loads_and_skips_malformed_lines(tmp_path):
    p = tmp_path / "t.txt"
    p.write_text("# comment\n"
                 "3 182 218 182 4 6  0 16 7  1.2 1.5\n"
                 "2 256 256 1 2 6  1 8 0  0.1 0.1\n"
                 "3 10 10 10 4 6  5 8 0  1 1\n"      # persistent must be 0 or 1
                 "3 10 10 10 4 6  0 12 0  1 1\n"     # tile rows must be 8, 16, -1, -2 or -3
                 "3 12 10 10 4 6  0 -2 4  1 1\n"
                 "garbage\n")
    try:
        assert synx.tuning_load(str(p)) == 3
        assert synx.tuning_path() == str(p)
    finally:
        synx.tuning_load(None)


def test_unreadable_table_is_an_error(tmp_path):
    try:
        try:
            synx.tuning_load(str(tmp_path / "missing.txt"))
            raise AssertionError("expected an error")
        except synx.SynxError:
            pass
    finally:
        synx.tuning_load(None)


def test_committed_table_parses_completely():
    path = os.path.join(ROOT, "ants_b200", "tuning_b200.txt")
    if not os.path.exists(path):
        return
    rows = [l for l in open(path) if l.strip() and not l.startswith("#")]
    try:
        assert synx.tuning_load(path) == len(rows) > 0
    finally:
        synx.tuning_load(None)
