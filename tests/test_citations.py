"""Every reference citation (``src/...jl:lines``) in this repository points at
lines that exist in the reference's files.  Needs the reference's sources;
skipped where they are not mounted."""

import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import check_citations  # noqa: E402


@pytest.mark.skipif(not os.path.isdir(check_citations.DEFAULT_REF), reason="reference sources not mounted")
def test_citations_point_inside_the_reference_files():
    total, bad = check_citations.check(REPO, check_citations.DEFAULT_REF)
    assert total > 100
    assert not bad, "\n".join(bad)
