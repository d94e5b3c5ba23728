"""LandmarkMap and its text loader (host only, no device).

The first three tests restate the reference's own unit tests in
crates/pf_core/src/landmark_map.rs:83-114 (add_has_at, parse_map_text,
parse_rejects_garbage); the others pin the loader's grammar as
landmark_map.rs:59-80 defines it: '#' comments, '[', ']', ':' and ','
read as spaces, exactly four numbers per line, the id parsed as f64 and cast
with Rust's saturating `as i32`, lines added as they are parsed."""
import numpy as np
import pytest

import cuda_pf_localization_b200 as pkg


@pytest.fixture
def m():
    lm = pkg.LandmarkMap()
    yield lm
    lm.close()


def test_add_has_at(m):
    assert not m.has(3)
    m.add(3, (1.0, 2.0, 3.0))
    assert m.has(3)
    assert m.at(3)[0] == pytest.approx(1.0)
    assert m.len_defined() == 1


def test_parse_map_text(m):
    n = m.load_from_str("# comment\n0: [1, 2, 3]\n5: [4.0, 5.0, 6.0]\n")
    assert n == 2
    assert m.has(0) and m.has(5)
    assert m.at(5)[2] == pytest.approx(6.0)


def test_parse_rejects_garbage(m):
    with pytest.raises(ValueError, match="line 1"):
        m.load_from_str("0 [1, 2]\n")


def test_capacity_counts_holes(m):
    m.add(7, (0.0, 0.0, 0.0))
    m.add(2, (1.0, 1.0, 1.0))
    assert m.capacity() == 8          # highest id + 1
    assert m.len_defined() == 2
    assert not m.has(3) and not m.has(-1) and not m.has(8)
    assert not m.is_empty()


def test_add_replaces(m):
    m.add(1, (1.0, 2.0, 3.0))
    m.add(1, (4.0, 5.0, 6.0))
    np.testing.assert_array_equal(m.at(1), [4.0, 5.0, 6.0])
    assert m.len_defined() == 1


def test_plain_format_comments_and_blank_lines(m):
    text = "\n   \n# header\n3 1.5 -2.5 1e-1  # trailing comment\n\r\n4: [0, 0, 0]\r\n"
    assert m.load_from_str(text) == 2
    np.testing.assert_array_equal(m.at(3), [1.5, -2.5, 0.1])
    assert m.has(4)


def test_id_parsed_as_float_and_truncated(m):
    # Rust: "2.9".parse::<f64>() as i32 == 2
    assert m.load_from_str("2.9: [1, 1, 1]\n") == 1
    assert m.has(2) and not m.has(3)


def test_lines_before_an_error_stay(m):
    with pytest.raises(ValueError, match="line 3"):
        m.load_from_str("0: [1, 2, 3]\n1: [4, 5, 6]\n2: [7, 8]\n3: [0, 0, 0]\n")
    assert m.has(0) and m.has(1)
    assert not m.has(2) and not m.has(3)


@pytest.mark.parametrize("bad", [
    "1: [a, 2, 3]",        # not a number
    "1: [0x10, 2, 3]",     # hexadecimal: Rust's f64 grammar rejects it
    "1: [1, 2, 3, 4]",     # five numbers
    "1 2 3",               # three numbers
    "1: [nan(1), 2, 3]",
])
def test_bad_lines_rejected(m, bad):
    with pytest.raises(ValueError):
        m.load_from_str(bad + "\n")


def test_negative_id_is_an_error(m):
    # the reference's add() asserts id >= 0 (a panic); here an error
    with pytest.raises(ValueError, match="non-negative"):
        m.load_from_str("-1: [1, 2, 3]\n")
    with pytest.raises(ValueError):
        m.add(-4, (0, 0, 0))
    assert m.len_defined() == 0


def test_at_absent_is_an_error(m):
    with pytest.raises(ValueError, match="not present"):
        m.at(0)


def test_rust_float_spellings(m):
    text = "0: [+1, -0.5, 2E2]\n1: [inf, -Infinity, NaN]\n"
    assert m.load_from_str(text) == 2
    np.testing.assert_array_equal(m.at(0), [1.0, -0.5, 200.0])
    a = m.at(1)
    assert a[0] == np.inf and a[1] == -np.inf and np.isnan(a[2])


def test_nan_id_casts_to_zero(m):
    # Rust's `f64::NAN as i32` is 0
    assert m.load_from_str("nan: [1, 2, 3]\n") == 1
    assert m.has(0)
