"""The table generator reproduces the committed headers (no hand edits)."""
import os

from awflcloud_b200 import gen_tables

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tables_header_is_generated():
    with open(os.path.join(HERE, "awflcloud_b200", "csrc", "awfl_tables.h")) as f:
        assert f.read() == gen_tables.emit_header()


def test_tv_header_is_generated():
    with open(os.path.join(HERE, "awflcloud_b200", "csrc", "awfl_tv.h")) as f:
        assert f.read() == gen_tables.emit_tv_header()


def test_tv_truncation_quirk():
    # integrate_poly keeps only the first n Taylor coefficients of (p^(d))^2, so the
    # n = 4 form has 39*a3^2 where the exact integral gives 39.1125*a3^2.
    terms = {(m, q): float(c) for m, q, c in gen_tables.tv_terms(4)}
    assert terms[(3, 3)] == 39.0
    terms5 = {(m, q): float(c) for m, q, c in gen_tables.tv_terms(5)}
    assert abs(terms5[(3, 3)] - 39.1125) < 1e-12
