"""The oracle reproduces its committed regression fixtures bit for bit
(tests/golden/oracle_fixtures.json, written by
tests/golden/make_oracle_fixtures.py): a change of the oracle's arithmetic
is caught here, and the device's FP64 form, bit-exact against the oracle in
tests/test_gpu_parity.py, is pinned to the same values."""
import json
import os

from tests.golden.make_oracle_fixtures import cases

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_matches_fixtures():
    with open(os.path.join(HERE, "golden", "oracle_fixtures.json")) as f:
        want = json.load(f)
    got = cases()
    assert sorted(got) == sorted(want)
    for name, w in want.items():
        g = got[name]
        for key, v in w.items():
            assert g[key] == v, (name, key)
