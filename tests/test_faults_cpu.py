"""Failures made on the host, checked without a GPU: a corrupt or truncated scattering table is refused by
the table reader with a clear error (the reference throws, NUTableInterpolation.cu:121)."""
import os

import pytest

from cudamonsel_b200 import data


def test_truncated_and_corrupt_tables_are_refused(tmp_path):
    src = data.si_tables()[0]
    text = open(src).read()
    cases = {"truncated": text[: len(text) // 2], "bad_dim": "7 " + text.split(None, 1)[1],
             "garbage": text.replace(text.split()[3], "x1x", 1), "empty": ""}
    for name, body in cases.items():
        p = tmp_path / (name + ".csv")
        p.write_text(body)
        with pytest.raises(ValueError, match="corrupt or truncated"):
            data.read_nu_table(str(p))
    dim, n, axes, vals = data.read_nu_table(src)  # the intact table still reads
    assert dim == 1 and vals.shape == tuple(n)
